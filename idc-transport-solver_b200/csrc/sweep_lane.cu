// Lane-pipelined sweep: host-side dispatch over degree, row-segment width, direction and second source,
// and the occupancy query.  The kernel is in sweep_lane_impl.cuh.
#include "sweep_lane_impl.cuh"

namespace idc {

namespace {

template <int P, bool ADJ, bool SRC2, bool PHI = false, typename TC = double>
cudaError_t launch_p(const SweepArgs &args, int grid, cudaStream_t stream) {
    switch (args.seg) {
        case 4: return lane::launch<P, 4, ADJ, SRC2, PHI, TC>(args, grid, stream);
        case 8: return lane::launch<P, 8, ADJ, SRC2, PHI, TC>(args, grid, stream);
        case 16: return lane::launch<P, 16, ADJ, SRC2, PHI, TC>(args, grid, stream);
        default: return cudaErrorInvalidValue;
    }
}

template <int P>
cudaError_t launch_dir(const SweepArgs &args, int grid, cudaStream_t stream, bool fp32) {
    if (fp32) {   // FP32 arithmetic: forward sweeps, with or without psi
        if (args.adjoint || args.src2) return cudaErrorInvalidValue;
        if (args.modal_src) {
            if (args.src || args.out || !args.phi_part) return cudaErrorInvalidValue;
            return launch_p<P, false, false, true, float>(args, grid, stream);
        }
        return launch_p<P, false, false, false, float>(args, grid, stream);
    }
    if (args.modal_src) {   // moments-only forward sweep
        if (args.adjoint || args.src2 || args.src || args.out || !args.phi_part) return cudaErrorInvalidValue;
        return launch_p<P, false, false, true>(args, grid, stream);
    }
    if (args.adjoint) return args.src2 ? cudaErrorInvalidValue : launch_p<P, true, false>(args, grid, stream);
    return args.src2 ? launch_p<P, false, true>(args, grid, stream) : launch_p<P, false, false>(args, grid, stream);
}

// Packed modal source of every interior (cell, quadrant) for the moments-only sweep (see idc_internal.hpp).
template <int P>
__global__ void modal_sources_kernel(GridDims g, const double *__restrict__ mom, double scale, double *__restrict__ out) {
    constexpr int N = P * P;
    const size_t total = (size_t)g.nx * g.ny * 4;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % 4);
        const size_t cell = t / 4;
        const int i = 1 + (int)(cell / g.ny), j = 1 + (int)(cell % g.ny);
        const size_t cidx = (size_t)i * (g.ny + 2) + j;
        double v[N], S[N];
#pragma unroll
        for (int m = 0; m < N; ++m) v[m] = mom ? scale * mom[cidx * N + m] : 0.0;
        const bool xn = k >= 2, yn = (k & 1) != 0;
#pragma unroll
        for (int m = 0; m < N; ++m) {   // the quadrant's sign flip x(d,e) -> sx^d sy^e x(d,e)
            const int d = m / P, e = m % P;
            if (((d & 1) && xn) != ((e & 1) && yn)) v[m] = -v[m];
        }
        modal_forward<P, false, false, double, false>(S, v);
        double *o = out + (cidx * 4 + k) * N;
#pragma unroll
        for (int m = 0; m < N; ++m) o[m] = S[m];
    }
}

// phi of the moments-only sweep: per interior cell and quadrant the fixed-order sum of its chunks' packed
// partials, transformed back and flipped, the quadrants added in order; ghost cells zero.
struct SlotBounds {
    int b[5];
};
template <int P>
__global__ void reduce_modal_partials_kernel(GridDims g, const double *__restrict__ part, SlotBounds sb, size_t stride,
                                             double *__restrict__ phi) {
    constexpr int N = P * P;
    const size_t total = (size_t)(g.nx + 2) * (g.ny + 2);
    for (size_t cidx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; cidx < total;
         cidx += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(cidx / (g.ny + 2)), j = (int)(cidx % (g.ny + 2));
        double acc[N];
#pragma unroll
        for (int m = 0; m < N; ++m) acc[m] = 0.0;
        if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) {
            for (int k = 0; k < 4; ++k) {
                if (sb.b[k + 1] == sb.b[k]) continue;
                double M[N], x[N];
#pragma unroll
                for (int m = 0; m < N; ++m) M[m] = 0.0;
                for (int sl = sb.b[k]; sl < sb.b[k + 1]; ++sl)
#pragma unroll
                    for (int m = 0; m < N; ++m) M[m] += part[(size_t)sl * stride + cidx * N + m];
                modal_backward<P, false, false, double, false>(x, M);
                const bool xn = k >= 2, yn = (k & 1) != 0;
#pragma unroll
                for (int m = 0; m < N; ++m) {
                    const int d = m / P, e = m % P;
                    acc[m] += (((d & 1) && xn) != ((e & 1) && yn)) ? -x[m] : x[m];
                }
            }
        }
#pragma unroll
        for (int m = 0; m < N; ++m) phi[cidx * N + m] = acc[m];
    }
}

int blocks_for(size_t n) {
    const size_t b = (n + 255) / 256;
    return (int)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

template <int P>
cudaError_t occ_p(int seg, bool src2, int *n) {
    switch (seg) {
        case 4: return src2 ? lane::occupancy<P, 4, false, true>(n) : lane::occupancy<P, 4, false, false>(n);
        case 8: return src2 ? lane::occupancy<P, 8, false, true>(n) : lane::occupancy<P, 8, false, false>(n);
        case 16: return src2 ? lane::occupancy<P, 16, false, true>(n) : lane::occupancy<P, 16, false, false>(n);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

bool sweep_lane_supports(int P, int precision, int seg) {
    return P >= 1 && P <= 3 && (precision == 0 || precision == 2) && (seg == 4 || seg == 8 || seg == 16);
}

int sweep_lane_warps() { return lane::kWarps; }

cudaError_t launch_sweep_lane(int P, int precision, const SweepArgs &args, int grid, cudaStream_t stream) {
    if (!args.trace || args.G > args.seg || args.R != 32 / args.seg) return cudaErrorInvalidValue;
    if (precision != 0 && precision != 2) return cudaErrorInvalidValue;
    const bool fp32 = precision == 2;
    switch (P) {
        case 1: return launch_dir<1>(args, grid, stream, fp32);
        case 2: return launch_dir<2>(args, grid, stream, fp32);
        case 3: return launch_dir<3>(args, grid, stream, fp32);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_modal_sources(const GridDims &g, const double *moments, double scale, double *out, cudaStream_t s) {
    const size_t n = (size_t)g.nx * g.ny * 4;
    switch (g.P) {
        case 1: modal_sources_kernel<1><<<blocks_for(n), 256, 0, s>>>(g, moments, scale, out); break;
        case 2: modal_sources_kernel<2><<<blocks_for(n), 256, 0, s>>>(g, moments, scale, out); break;
        case 3: modal_sources_kernel<3><<<blocks_for(n), 256, 0, s>>>(g, moments, scale, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_reduce_modal_partials(const GridDims &g, const double *part, const int slot_begin[5], size_t stride,
                                         double *phi, cudaStream_t s) {
    SlotBounds sb;
    for (int k = 0; k < 5; ++k) sb.b[k] = slot_begin[k];
    const size_t n = (size_t)(g.nx + 2) * (g.ny + 2);
    switch (g.P) {
        case 1: reduce_modal_partials_kernel<1><<<blocks_for(n), 256, 0, s>>>(g, part, sb, stride, phi); break;
        case 2: reduce_modal_partials_kernel<2><<<blocks_for(n), 256, 0, s>>>(g, part, sb, stride, phi); break;
        case 3: reduce_modal_partials_kernel<3><<<blocks_for(n), 256, 0, s>>>(g, part, sb, stride, phi); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

namespace {
template <int P>
cudaError_t launch_batched_p(int seg, const SweepArgs &args, const SweepArgs *table, int grid, cudaStream_t stream) {
    switch (seg) {
        case 4: return lane::launch_batched<P, 4>(args, table, grid, stream);
        case 8: return lane::launch_batched<P, 8>(args, table, grid, stream);
        case 16: return lane::launch_batched<P, 16>(args, table, grid, stream);
        default: return cudaErrorInvalidValue;
    }
}
template <int P>
cudaError_t occupancy_batched_p(int seg, int *n) {
    switch (seg) {
        case 4: return lane::occupancy_batched<P, 4>(n);
        case 8: return lane::occupancy_batched<P, 8>(n);
        case 16: return lane::occupancy_batched<P, 16>(n);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace

cudaError_t launch_sweep_lane_batched(int P, const SweepArgs &args, const SweepArgs *table, int grid,
                                      cudaStream_t stream) {
    if (args.G > args.seg || args.R != 32 / args.seg || !table) return cudaErrorInvalidValue;
    switch (P) {
        case 1: return launch_batched_p<1>(args.seg, args, table, grid, stream);
        case 2: return launch_batched_p<2>(args.seg, args, table, grid, stream);
        case 3: return launch_batched_p<3>(args.seg, args, table, grid, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t sweep_lane_batched_occupancy(int P, int seg, int *blocks_per_sm) {
    switch (P) {
        case 1: return occupancy_batched_p<1>(seg, blocks_per_sm);
        case 2: return occupancy_batched_p<2>(seg, blocks_per_sm);
        case 3: return occupancy_batched_p<3>(seg, blocks_per_sm);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t sweep_lane_occupancy(int P, int seg, bool src2, int *blocks_per_sm) {
    switch (P) {
        case 1: return occ_p<1>(seg, src2, blocks_per_sm);
        case 2: return occ_p<2>(seg, src2, blocks_per_sm);
        case 3: return occ_p<3>(seg, src2, blocks_per_sm);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace idc
