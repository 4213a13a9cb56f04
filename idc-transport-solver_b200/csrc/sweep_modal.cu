// Modal sweep: host-side dispatch over degree, precision, row-segment width and direction, the shared-
// memory size, and the inflow-trace kernel.  The kernels are in sweep_modal_impl.cuh.
#include "sweep_modal_impl.cuh"

#include <algorithm>

IDC_MODAL_LAUNCHERS(extern, 0, false)
IDC_MODAL_LAUNCHERS(extern, 0, true)
IDC_MODAL_LAUNCHERS(extern, 1, false)
IDC_MODAL_LAUNCHERS(extern, 1, true)
IDC_MODAL_LAUNCHERS(extern, 2, false)
IDC_MODAL_BATCHED(extern, 0)
IDC_MODAL_BATCHED(extern, 1)

namespace idc {

namespace {

using modal::kS;
using modal::prefetch_depth;

// Inflow traces of the ghost cells, one thread per (boundary position k, ordinate q):
// k < nx: the y trace g(d) = sum_e x'(d,e) of the ghost cell below column k (sweep order);
// k >= nx: the x trace f(e) = sum_d x'(d,e) of the ghost cell left of row k - nx (sweep order);
// x' is the sign-flipped ghost source, and the traces are packed modal (Wp h) unless MODAL is false.
template <int P, bool MODAL>
__global__ void inflow_traces_kernel(const double *src, const double *xi, const double *eta, int nx, int ny, int nq,
                                     double *out) {
    constexpr int N = P * P;
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)(nx + ny) * nq) return;
    const int k = (int)(idx / nq), q = (int)(idx % nq);
    const bool xneg = xi[q] < 0, yneg = eta[q] < 0;
    int i, j;
    if (k < nx) {
        i = xneg ? nx - k : 1 + k;
        j = yneg ? ny + 1 : 0;
    } else {
        i = xneg ? nx + 1 : 0;
        j = yneg ? ny - (k - nx) : 1 + (k - nx);
    }
    const double *v = src + (((size_t)i * (ny + 2) + j) * nq + q) * N;
    double h[P];
#pragma unroll
    for (int m = 0; m < P; ++m) h[m] = 0.0;
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e) {
            const double sgn = ((xneg && (d & 1)) != (yneg && (e & 1))) ? -1.0 : 1.0;
            const double val = sgn * v[e + P * d];
            if (k < nx)
                h[d] += val;
            else
                h[e] += val;
        }
    double* o = out + idx * P;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        if (MODAL) {
            double acc = 0.0;
#pragma unroll
            for (int n = 0; n < P; ++n) acc = fma(ModalTable<P>::W(m, n), h[n], acc);
            o[m] = acc;
        } else {
            o[m] = h[m];
        }
    }
}

// Batched forms of the inflow-trace kernel and of the moment reduction: one launch for every problem of
// a batched sweep (blockIdx.y = problem), reading the problems' arrays from the launch's SweepArgs table.
template <int P, bool MODAL>
__global__ void inflow_traces_batched_kernel(const SweepArgs *__restrict__ table) {
    const SweepArgs &a = table[blockIdx.y];
    if (!a.src || !a.inflow) return;
    constexpr int N = P * P;
    const int nx = a.nx, ny = a.ny, nq = a.nq;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < (size_t)(nx + ny) * nq;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(idx / nq), q = (int)(idx % nq);
        const bool xneg = a.xi[q] < 0, yneg = a.eta[q] < 0;
        int i, j;
        if (k < nx) {
            i = xneg ? nx - k : 1 + k;
            j = yneg ? ny + 1 : 0;
        } else {
            i = xneg ? nx + 1 : 0;
            j = yneg ? ny - (k - nx) : 1 + (k - nx);
        }
        const double *v = a.src + (((size_t)i * (ny + 2) + j) * nq + q) * N;
        double h[P];
#pragma unroll
        for (int m = 0; m < P; ++m) h[m] = 0.0;
#pragma unroll
        for (int d = 0; d < P; ++d)
#pragma unroll
            for (int e = 0; e < P; ++e) {
                const double sgn = ((xneg && (d & 1)) != (yneg && (e & 1))) ? -1.0 : 1.0;
                const double val = sgn * v[e + P * d];
                if (k < nx)
                    h[d] += val;
                else
                    h[e] += val;
            }
        double *o = const_cast<double *>(a.inflow) + idx * P;   // the batch owns these trace buffers
#pragma unroll
        for (int m = 0; m < P; ++m) {
            if (MODAL) {
                double acc = 0.0;
#pragma unroll
                for (int n = 0; n < P; ++n) acc = fma(ModalTable<P>::W(m, n), h[n], acc);
                o[m] = acc;
            } else {
                o[m] = h[m];
            }
        }
    }
}

// phi = sum of the problem's partial-moment slots (fixed order), ghost cells zero; phi is the table's `phi`.
__global__ void reduce_partials_batched_kernel(const SweepArgs *__restrict__ table, int N) {
    const SweepArgs &a = table[blockIdx.y];
    if (!a.phi || !a.phi_part) return;
    const size_t total = (size_t)(a.nx + 2) * (a.ny + 2) * N;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t cell = t / N;
        const int i = (int)(cell / (a.ny + 2)), j = (int)(cell % (a.ny + 2));
        double acc = 0.0;
        if (i >= 1 && i <= a.nx && j >= 1 && j <= a.ny)
            for (int sl = 0; sl < a.phi_slots; ++sl) acc += a.phi_part[(size_t)sl * a.phi_slot_stride + t];
        a.phi[t] = acc;
    }
}

template <int P, int MODE, bool ADJ>
cudaError_t launch_dir(const SweepArgs &args, int grid, size_t smem, cudaStream_t stream) {
    switch (args.seg) {
        case 4: return modal::launch_seg<P, MODE, 4, ADJ>(args, grid, smem, stream);
        case 8: return modal::launch_seg<P, MODE, 8, ADJ>(args, grid, smem, stream);
        case 16: return modal::launch_seg<P, MODE, 16, ADJ>(args, grid, smem, stream);
        case 32: return modal::launch_seg<P, MODE, 32, ADJ>(args, grid, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

// The transposed sweep exists for the FP64 and refined modes.
template <int P, int MODE>
cudaError_t launch_t(const SweepArgs &args, int grid, size_t smem, cudaStream_t stream) {
    if (!args.adjoint) return launch_dir<P, MODE, false>(args, grid, smem, stream);
    if constexpr (MODE == 2) return cudaErrorInvalidValue;
    else return launch_dir<P, MODE, true>(args, grid, smem, stream);
}

template <int P, int MODE>
cudaError_t occ_t(int seg, int threads, size_t smem, int *n) {
    switch (seg) {
        case 4: return modal::occ_seg<P, MODE, 4, false>(threads, smem, n);
        case 8: return modal::occ_seg<P, MODE, 8, false>(threads, smem, n);
        case 16: return modal::occ_seg<P, MODE, 16, false>(threads, smem, n);
        case 32: return modal::occ_seg<P, MODE, 32, false>(threads, smem, n);
        default: return cudaErrorInvalidValue;
    }
}

template <int P, bool MODAL>
cudaError_t inflow_t(const double *src, const double *xi, const double *eta, int nx, int ny, int nq, double *out,
                     cudaStream_t stream) {
    const size_t n = (size_t)(nx + ny) * nq;
    const int block = 128;
    inflow_traces_kernel<P, MODAL><<<(unsigned)((n + block - 1) / block), block, 0, stream>>>(src, xi, eta, nx, ny,
                                                                                             nq, out);
    return cudaGetLastError();
}

template <int P, int MODE>
cudaError_t launch_batched_t(const SweepArgs &launch, const SweepArgs *table, int grid, size_t smem,
                             cudaStream_t stream) {
    switch (launch.seg) {
        case 4: return modal::launch_seg_batched<P, MODE, 4>(launch, table, grid, smem, stream);
        case 8: return modal::launch_seg_batched<P, MODE, 8>(launch, table, grid, smem, stream);
        case 16: return modal::launch_seg_batched<P, MODE, 16>(launch, table, grid, smem, stream);
        case 32: return modal::launch_seg_batched<P, MODE, 32>(launch, table, grid, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

template <int P>
size_t smem_p(int precision, int wn, int G, int seg) {
    const int na = modal::aux_per_compute(P, wn), D = prefetch_depth(P), rw = 32 / seg;
    switch (precision) {
        case 0: return modal::layout_bytes(wn, na, G, P, D, rw, modal::slot_words<P, 0>());
        case 1: return modal::layout_bytes(wn, na, G, P, D, rw, modal::slot_words<P, 1>());
        default: return modal::layout_bytes(wn, na, G, P, D, rw, modal::slot_words<P, 2>());
    }
}

size_t sweep_modal_src2_bytes(int P, int wn) {
    switch (P) {
        case 1: return modal::src2_layout_bytes(wn, modal::aux_per_compute(1, wn), 1, prefetch_depth(1));
        case 2: return modal::src2_layout_bytes(wn, modal::aux_per_compute(2, wn), 2, prefetch_depth(2));
        default: return modal::src2_layout_bytes(wn, modal::aux_per_compute(3, wn), 3, prefetch_depth(3));
    }
}

size_t sweep_modal_smem_bytes(int P, int precision, int wn, int G, int seg) {
    switch (P) {
        case 1: return smem_p<1>(precision, wn, G, seg);
        case 2: return smem_p<2>(precision, wn, G, seg);
        default: return smem_p<3>(precision, wn, G, seg);
    }
}

int sweep_modal_threads(int P, int wn) { return modal::cta_warps(P, wn) * 32; }

// 4 compute warps with 2 aux warps each (13 warps): measured fastest on B200 at Q1 and Q2, S4..S16
int sweep_modal_default_wn(int) { return 4; }

int sweep_modal_fit_wn(int P, int precision, int wn, int G, int seg) {
    int dev = 0, limit = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        limit = 227 * 1024;
    wn = std::min(wn, modal::max_compute_warps(P));
    while (wn > 1 && sweep_modal_smem_bytes(P, precision, wn, G, seg) > (size_t)limit) --wn;
    return wn;
}

int sweep_modal_max_wn(int P) { return modal::max_compute_warps(P); }

#define IDC_MDISPATCH(P_, FN, ...)             \
    switch (precision) {                       \
        case 0: return FN<P_, 0>(__VA_ARGS__); \
        case 1: return FN<P_, 1>(__VA_ARGS__); \
        case 2: return FN<P_, 2>(__VA_ARGS__); \
        default: return cudaErrorInvalidValue; \
    }

cudaError_t launch_sweep_modal(int P, int precision, const SweepArgs &args, int grid, size_t smem,
                               cudaStream_t stream) {
    if (args.wn < 1 || args.wn > sweep_modal_max_wn(P) || !args.trace || args.seg < 4 || args.seg > 32 ||
        (args.seg & (args.seg - 1)) || args.G > args.seg)
        return cudaErrorInvalidValue;
    switch (P) {
        case 1: IDC_MDISPATCH(1, launch_t, args, grid, smem, stream);
        case 2: IDC_MDISPATCH(2, launch_t, args, grid, smem, stream);
        case 3: IDC_MDISPATCH(3, launch_t, args, grid, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_sweep_modal_batched(int P, int precision, const SweepArgs &launch, const SweepArgs *table, int grid,
                                       size_t smem, cudaStream_t stream) {
    if (launch.wn < 1 || launch.wn > sweep_modal_max_wn(P) || launch.seg < 4 || launch.seg > 32 || (launch.seg & (launch.seg - 1)) ||
        launch.G > launch.seg || !table || launch.adjoint)
        return cudaErrorInvalidValue;
    if (precision != 0 && precision != 1) return cudaErrorInvalidValue;
    switch (P) {
        case 1: return precision == 0 ? launch_batched_t<1, 0>(launch, table, grid, smem, stream)
                                      : launch_batched_t<1, 1>(launch, table, grid, smem, stream);
        case 2: return precision == 0 ? launch_batched_t<2, 0>(launch, table, grid, smem, stream)
                                      : launch_batched_t<2, 1>(launch, table, grid, smem, stream);
        case 3: return precision == 0 ? launch_batched_t<3, 0>(launch, table, grid, smem, stream)
                                      : launch_batched_t<3, 1>(launch, table, grid, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batched_helpers(int P, bool modal_inflow, const SweepArgs *table, int members, bool inflow,
                                   bool reduce, cudaStream_t stream) {
    if (members < 1 || members > 65535) return cudaErrorInvalidValue;
    const dim3 grid(148, (unsigned)members), block(128);
    if (inflow) {
        switch (P) {
            case 1: modal_inflow ? inflow_traces_batched_kernel<1, true><<<grid, block, 0, stream>>>(table)
                                 : inflow_traces_batched_kernel<1, false><<<grid, block, 0, stream>>>(table); break;
            case 2: modal_inflow ? inflow_traces_batched_kernel<2, true><<<grid, block, 0, stream>>>(table)
                                 : inflow_traces_batched_kernel<2, false><<<grid, block, 0, stream>>>(table); break;
            case 3: modal_inflow ? inflow_traces_batched_kernel<3, true><<<grid, block, 0, stream>>>(table)
                                 : inflow_traces_batched_kernel<3, false><<<grid, block, 0, stream>>>(table); break;
            default: return cudaErrorInvalidValue;
        }
    }
    if (reduce) reduce_partials_batched_kernel<<<dim3(148, (unsigned)members), 256, 0, stream>>>(table, P * P);
    return cudaGetLastError();
}

cudaError_t sweep_modal_occupancy(int P, int precision, int seg, int threads, size_t smem, int *blocks_per_sm) {
    switch (P) {
        case 1: IDC_MDISPATCH(1, occ_t, seg, threads, smem, blocks_per_sm);
        case 2: IDC_MDISPATCH(2, occ_t, seg, threads, smem, blocks_per_sm);
        case 3: IDC_MDISPATCH(3, occ_t, seg, threads, smem, blocks_per_sm);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_inflow_traces(int P, bool modal, const double *src, const double *xi, const double *eta, int nx,
                                 int ny, int nq, double *out, cudaStream_t stream) {
    switch (P) {
        case 1: return modal ? inflow_t<1, true>(src, xi, eta, nx, ny, nq, out, stream)
                             : inflow_t<1, false>(src, xi, eta, nx, ny, nq, out, stream);
        case 2: return modal ? inflow_t<2, true>(src, xi, eta, nx, ny, nq, out, stream)
                             : inflow_t<2, false>(src, xi, eta, nx, ny, nq, out, stream);
        case 3: return modal ? inflow_t<3, true>(src, xi, eta, nx, ny, nq, out, stream)
                             : inflow_t<3, false>(src, xi, eta, nx, ny, nq, out, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace idc
