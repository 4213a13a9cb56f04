// Batched sweeps of independent problems in one persistent launch per DG degree (batch.cpp).
#pragma once

#include "context.hpp"

#include <map>
#include <utility>
#include <vector>

namespace idc {

class Batch {
public:
    ~Batch();
    Status add(Context *c);
    // per problem p (arrays indexed like `members`, entries nullable): outs[p] <- L^{-1}(srcs[p] +
    // scale phi_sc[p]), phis[p] <- P outs[p]; device pointers.  phi_sc[p] holds the scattering moments
    // sigma_s phi / (4 pi) per cell (launch_scatter_moments), S phi without the ordinate broadcast
    Status sweep(const double *const *srcs, double *const *outs, const double *const *phi_sc, double scale,
                 double *const *phis, double dt, int precision, const std::vector<char> *active = nullptr);
    // GMRES(restart) on every member's Peierls system at once (the algorithm of Context::gmres_peierls, with
    // each member's preconditioner): every Krylov step sweeps all unconverged members in one batched sweep,
    // their Arnoldi steps and DSA applications run on the device per member, with one host synchronisation
    // per step for all.  psi_inout[p]: Q on entry, psi on return (device).  iters / resids: per member.
    Status gmres_solve(double *const *psi_inout, double dt, double abs_tol, int restart, int64_t max_its,
                       int precision, int64_t *iters, double *resids);
    // times the candidate tile shapes per degree on the given inputs and keeps the fastest
    Status autotune(const double *const *srcs, double *const *outs, double dt, int precision);
    // the tile shape used for degree P at `precision` (set: seg in {4,8,16,32}, wn in 1..7; 0, 0 = default)
    Status set_shape(int P, int precision, int seg, int wn);
    void get_shape(int P, int precision, int *seg, int *wn) const;

    std::vector<Context *> members;
    std::map<std::pair<int, int>, std::pair<int, int>> tuned;   // (P, precision) -> (seg, wn)
    float last_ms = 0.f;

private:
    struct Group {
        int P = 0, seg = 0, wn = 0, G = 0, precision = -1, n_items = 0, grid = 0;
        size_t smem = 0;
        std::vector<int> members, items_per_rb;
        SweepItem *d_items = nullptr;
        int *d_sync = nullptr;
        SweepArgs *d_table = nullptr;
        SweepArgs *h_table = nullptr;            // pinned: uploads do not synchronise the stream
        std::vector<SweepArgs> uploaded;         // the table on the device (re-uploaded only on change)
        cudaEvent_t upload_done = nullptr;       // the last upload has read h_table
        std::vector<double *> trace, phi_part, inflow;
        std::vector<size_t> trace_len;
    };
    Status build_group(Group &g, int precision);
    Status launch_group(Group &g, const double *const *srcs, double *const *outs, const double *const *phi_sc,
                        double scale, double *const *phis, double dt, const std::vector<char> *active);
    void release();
    // every group launches on the first member's stream, so that one synchronisation and one event pair
    // cover the whole batched sweep
    cudaStream_t stream() const { return members[0]->stream; }
    std::vector<Group> groups;
};

}  // namespace idc
