// Lane-pipelined sweep: host-side dispatch over degree, row-segment width, direction and second source,
// and the occupancy query.  The kernel is in sweep_lane_impl.cuh.
#include "sweep_lane_impl.cuh"

namespace idc {

namespace {

template <int P, bool ADJ, bool SRC2>
cudaError_t launch_p(const SweepArgs &args, int grid, cudaStream_t stream) {
    switch (args.seg) {
        case 4: return lane::launch<P, 4, ADJ, SRC2>(args, grid, stream);
        case 8: return lane::launch<P, 8, ADJ, SRC2>(args, grid, stream);
        case 16: return lane::launch<P, 16, ADJ, SRC2>(args, grid, stream);
        default: return cudaErrorInvalidValue;
    }
}

template <int P>
cudaError_t launch_dir(const SweepArgs &args, int grid, cudaStream_t stream) {
    if (args.adjoint) return args.src2 ? cudaErrorInvalidValue : launch_p<P, true, false>(args, grid, stream);
    return args.src2 ? launch_p<P, false, true>(args, grid, stream) : launch_p<P, false, false>(args, grid, stream);
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
    return P >= 1 && P <= 3 && precision == 0 && (seg == 4 || seg == 8 || seg == 16);
}

int sweep_lane_warps() { return lane::kWarps; }

cudaError_t launch_sweep_lane(int P, const SweepArgs &args, int grid, cudaStream_t stream) {
    if (!args.trace || args.G > args.seg || args.R != 32 / args.seg) return cudaErrorInvalidValue;
    switch (P) {
        case 1: return launch_dir<1>(args, grid, stream);
        case 2: return launch_dir<2>(args, grid, stream);
        case 3: return launch_dir<3>(args, grid, stream);
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
