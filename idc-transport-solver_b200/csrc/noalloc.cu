// idc_sweep_noalloc: the sweep for callers that cannot allocate device memory.
//
// Who needs it: a host code that owns all of the GPU's memory through its own arena (large simulation
// codes often reserve most of HBM at start-up and forbid allocations outside it), and loops that cannot
// afford cudaMalloc / cudaFree, which may synchronise the device and can fail once memory is reserved.
// Such a caller passes every input and output as a device pointer it already owns; the only other
// memory the sweep needs -- its work-queue head, device error word, per-item progress flags and the
// work-item list -- lives in the fixed file-scope array below instead of in a context-owned buffer.
//
// The array is a static __device__ object: every GPU that loads this library holds it (about 96 KiB)
// until the process exits.  Its host-side name is only a stand-in, so its device address is looked up
// once per device with cudaGetSymbolAddress, with that device current, on the first call on that device.
//
// The sweep runs without fused moments; phi_out is formed afterwards by the moment kernel of idc_pmv,
// which adds the ordinates of each (cell, dof) in index order, so phi_out repeats bitwise from call to
// call (the row-synchronous kernel's fused moments would add across thread blocks with atomics).  The
// call reads the ordinates back to the host and synchronises `stream` before it returns.
#include "idc_internal.hpp"
#include "idcsweep.h"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

namespace {

constexpr int kMaxItems = IDC_NOALLOC_MAX_ITEMS;
constexpr int kMaxOrdinates = IDC_NOALLOC_MAX_ORDINATES;
constexpr int kMaxDevices = 64;
// [0] queue head, [1] error word, [2, 2 + kMaxItems) progress flags, then the work items
constexpr int kItemInts = (int)(sizeof(idc::SweepItem) / sizeof(int));
constexpr int kScratchInts = 2 + kMaxItems + kMaxItems * kItemInts;
static_assert(sizeof(idc::SweepItem) % sizeof(int) == 0, "SweepItem must be a whole number of ints");

static __device__ __align__(256) int g_sweep_scratch[kScratchInts];

std::mutex g_lock;                        // one call at a time per process: the array is shared
int *g_scratch_addr[kMaxDevices] = {};    // device address of g_sweep_scratch, per device
idc::SweepItem g_items_host[kMaxItems];   // staging for the item list (host, static)
double g_xi_host[kMaxOrdinates], g_eta_host[kMaxOrdinates];

// The status code is returned; its text goes to idc_last_error_message() as for every other entry point.
int fail(int code, const std::string &m) {
    idc::set_last_error(m);
    return code;
}

// Restores the caller's current device on every exit path.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() { cudaGetDevice(&prev); }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int idc_sweep_noalloc(const idc_problem_desc *desc, int64_t nq, const double *xi, const double *eta,
                                 const double *w, const int64_t quad_bounds[5], const double *sigma_t,
                                 const double *source, double *result, double dt, double *phi_out, int precision,
                                 void *stream_ptr) {
    if (!desc || !xi || !eta || !w || !quad_bounds || !sigma_t || !source || !result)
        return fail(IDC_ERR_ARG, "idc_sweep_noalloc: null argument");
    if (desc->nx < 1 || desc->ny < 1 || desc->nx > (1 << 20) || desc->ny > (1 << 20))
        return fail(IDC_ERR_ARG, "idc_sweep_noalloc: bad grid size");
    if (!(desc->bx > desc->ax) || !(desc->by > desc->ay)) return fail(IDC_ERR_ARG, "idc_sweep_noalloc: empty domain");
    if (desc->dg_degree < 0 || desc->dg_degree > 2 || desc->sigma_degree != 0 || desc->flags != 0)
        return fail(IDC_ERR_UNSUPPORTED, "idc_sweep_noalloc: DG degree 0..2 and piecewise-constant sigma only");
    if (precision < 0 || precision > 2) return fail(IDC_ERR_ARG, "idc_sweep_noalloc: unknown precision");
    if (!(dt > 0)) return fail(IDC_ERR_ARG, "idc_sweep_noalloc: dt must be positive (+inf for steady state)");
    if (nq < 1 || nq > kMaxOrdinates)
        return fail(IDC_ERR_ARG, "idc_sweep_noalloc: nq must be in 1.." + std::to_string(kMaxOrdinates));
    if (quad_bounds[0] != 0 || quad_bounds[4] != nq) return fail(IDC_ERR_ARG, "idc_sweep_noalloc: bad quad_bounds");
    for (int k = 0; k < 4; ++k)
        if (quad_bounds[k + 1] < quad_bounds[k]) return fail(IDC_ERR_ARG, "idc_sweep_noalloc: bad quad_bounds");

    const int P = (int)desc->dg_degree + 1;
    const int64_t nx = desc->nx, ny = desc->ny;

    // tile shape: the same automatic choice as the context-based entry points
    int qmax = 0;
    for (int k = 0; k < 4; ++k) qmax = std::max<int>(qmax, (int)(quad_bounds[k + 1] - quad_bounds[k]));
    int G = std::min(qmax, P == 3 ? 36 : 64);
    int R = std::max(1, std::min(16, 320 / G));
    if (R > ny) R = (int)ny;
    const int nrb = (int)((ny + R - 1) / R);
    int per_rb = 0;
    for (int k = 0; k < 4; ++k) {
        const int cnt = (int)(quad_bounds[k + 1] - quad_bounds[k]);
        per_rb += cnt == 0 ? 0 : (cnt + G - 1) / G;
    }
    if ((int64_t)nrb * per_rb > kMaxItems)
        return fail(IDC_ERR_ARG, "idc_sweep_noalloc: problem needs " + std::to_string((int64_t)nrb * per_rb) +
                                     " work items, more than the fixed scratch holds (" + std::to_string(kMaxItems) +
                                     "); use idc_sweep");

    if (desc->device < 0 || desc->device >= kMaxDevices) return fail(IDC_ERR_ARG, "idc_sweep_noalloc: device ordinal");

    std::lock_guard<std::mutex> lock(g_lock);
    DeviceGuard guard;
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    cudaError_t e = cudaSetDevice(desc->device);
    if (e != cudaSuccess) return fail(IDC_ERR_ARG, std::string("idc_sweep_noalloc: cudaSetDevice: ") + cudaGetErrorString(e));

    // once per device, with that device current: the device address of the scratch array
    int *scratch = g_scratch_addr[desc->device];
    if (!scratch) {
        e = cudaGetSymbolAddress((void **)&scratch, g_sweep_scratch);
        if (e != cudaSuccess || !scratch)
            return fail(IDC_ERR_CUDA, std::string("idc_sweep_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_addr[desc->device] = scratch;
    }

    // ordinate signs must match their quadrants (OrdinateSet::SetSigns)
    e = cudaMemcpyAsync(g_xi_host, xi, sizeof(double) * nq, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g_eta_host, eta, sizeof(double) * nq, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(IDC_ERR_CUDA, std::string("idc_sweep_noalloc: reading ordinates: ") + cudaGetErrorString(e));
    for (int k = 0; k < 4; ++k)
        for (int64_t q = quad_bounds[k]; q < quad_bounds[k + 1]; ++q) {
            const bool xneg = k >= 2, yneg = (k & 1) != 0;
            if ((xneg ? !(g_xi_host[q] < 0) : !(g_xi_host[q] > 0)) || (yneg ? !(g_eta_host[q] < 0) : !(g_eta_host[q] > 0)))
                return fail(IDC_ERR_ARG, "idc_sweep_noalloc: ordinate " + std::to_string(q) + " outside its quadrant");
        }

    // work items, row-block major (same schedule as the context-based sweep)
    int n = 0, prev_first = -1;
    for (int rb = 0; rb < nrb; ++rb) {
        const int first = n;
        int slot = 0;
        for (int k = 0; k < 4; ++k) {
            const int cnt = (int)(quad_bounds[k + 1] - quad_bounds[k]);
            if (cnt == 0) continue;
            const int nch = (cnt + G - 1) / G;
            int beg = (int)quad_bounds[k];
            for (int c = 0; c < nch; ++c, ++slot) {
                const int sz = cnt / nch + (c < cnt % nch ? 1 : 0);
                g_items_host[n++] = idc::SweepItem{k, beg, sz, rb, rb == 0 ? -1 : prev_first + slot};
                beg += sz;
            }
        }
        prev_first = first;
    }
    int *head = scratch, *err_word = scratch + 1, *progress = scratch + 2;
    auto *items = reinterpret_cast<idc::SweepItem *>(scratch + 2 + kMaxItems);

    int sms = 0, per_sm = 0;
    const int block = ((G * R + 31) / 32) * 32;
    const size_t smem = idc::sweep_smem_bytes(P, R, G);
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, desc->device);
    if (e == cudaSuccess) e = idc::sweep_occupancy(P, precision, block, smem, &per_sm);
    if (e != cudaSuccess || per_sm < 1)
        return fail(IDC_ERR_CUDA, std::string("idc_sweep_noalloc: occupancy: ") + cudaGetErrorString(e));

    // the array keeps the last call's contents: clear head, error word and progress flags
    e = cudaMemcpyAsync(items, g_items_host, sizeof(idc::SweepItem) * n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch, 0, sizeof(int) * (2 + (size_t)n), stream);
    if (e != cudaSuccess) return fail(IDC_ERR_CUDA, std::string("idc_sweep_noalloc: staging: ") + cudaGetErrorString(e));

    idc::SweepArgs a{};
    a.src = source;
    a.out = result;
    a.sigma_t = sigma_t;
    a.sigma_s = nullptr;
    a.phi_scatter = nullptr;
    a.scatter_scale = 1.0;
    a.phi = nullptr;   // phi_out is formed after the sweep, in a fixed order
    a.xi = xi;
    a.eta = eta;
    a.w = w;
    a.nx = (int)nx;
    a.ny = (int)ny;
    a.nq = (int)nq;
    a.dx = (desc->bx - desc->ax) / (double)nx;
    a.dy = (desc->by - desc->ay) / (double)ny;
    a.inv_dt = 1.0 / dt;
    a.items = items;
    a.n_items = n;
    a.R = R;
    a.G = G;
    a.n_refine = 1;
    a.next_item = head;
    a.error = err_word;
    a.progress = progress;
    a.spin_limit = 1ll << 22;
    e = idc::launch_sweep(P, precision, a, std::min(n, per_sm * sms), block, smem, stream);
    if (e != cudaSuccess) return fail(IDC_ERR_CUDA, std::string("idc_sweep_noalloc: sweep: ") + cudaGetErrorString(e));
    if (phi_out) {   // phi = sum_q w_q psi_q on interior cells in index order (TransportOperator::Pmv), ghosts 0
        const idc::GridDims g{(int)nx, (int)ny, (int)nq, P, a.dx, a.dy};
        e = idc::launch_zero_ghost_phi(g, phi_out, stream);
        if (e == cudaSuccess) e = idc::launch_pmv(g, 1.0, 0.0, w, result, phi_out, stream);
        if (e != cudaSuccess)
            return fail(IDC_ERR_CUDA, std::string("idc_sweep_noalloc: moments: ") + cudaGetErrorString(e));
    }
    // the error word comes back on the caller's stream, behind the sweep (a legacy-stream copy would also
    // wait for the caller's other blocking streams)
    int dev_err = 0;
    e = cudaMemcpyAsync(&dev_err, err_word, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(IDC_ERR_CUDA, std::string("idc_sweep_noalloc: sweep: ") + cudaGetErrorString(e));
    if (dev_err != idc::kDevOk)
        return fail(IDC_ERR_TIMEOUT, "idc_sweep_noalloc: a device-side wait gave up; the result is not valid");
    return IDC_OK;
}
