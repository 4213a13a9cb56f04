// Per-cell arithmetic of the upwind-DG sweep in the packed modal basis of the 1-D upwind matrix.
//
// The reference solves each (cell, ordinate) system A x = B by Gaussian elimination
// (SweepCellSolveBase::ConstructAndSolve -> CalcB / CalcA / GE, linear_solvers/RKDG/SweepCellSolve/
// SweepCellSolve.hpp:312-353, SweepLinearSolveSpec.cpp:511-640).  The matrix has Kronecker structure,
//     A = dy xi (Mx (x) I) + dx eta (I (x) My) + (sigma_t + 1/dt) dx dy I,
// and the upwind coupling of B is rank one per face: B(d,e) += dy xi R(d,a) psi_up(a,e) with
// R(d,a) = u_d * const.  After the quadrant's sign flip x(d,e) -> sx^d sy^e x(d,e) (sx = -1 for
// xi < 0, sy = -1 for eta < 0) and division by dx dy, every quadrant reads
//     A' = ax (M (x) I) + ay (I (x) M) + s I,   ax = |xi|/dx, ay = |eta|/dy, s = sigma_t + 1/dt,
//     B' = src' + ax u (x) f + ay g (x) u,      u_d = (-1)^d (2d+1),
// where f(e) = sum_d x'_left(d,e) and g(d) = sum_e x'_below(d,e) are the face traces of the upwind
// neighbours (the ghost cells' traces on the inflow boundary).  In the packed basis Vp (x) Vp of
// modal_tables.h, A' is block diagonal (blocks of 1, 2 and 4 reals that are complex divisions), so
//     Z = blocks^-1 (Wp src' Wp^T + ax uh (x) fh + ay gh (x) uh),  fh = Wp f, gh = Wp g,
// and the neighbours' traces in the same basis are plain sums of Z's coefficients:
//     fh_out(b) = sum_a t_a Z(a,b), gh_out(a) = sum_b t_b Z(a,b), t = (1, 0, ..., 1).
// x' = Vp Z Vp^T is needed only for the stored psi and the moments.  The recurrence from cell to
// cell is therefore a handful of fused multiply-adds deep, and the dense transforms are off it.
//
// The transposed (adjoint) sweep solves A'^T lam = r + ax 1 (x) ft + ay gt (x) 1 with the outgoing traces
// ft(e) = sum_d u_d lam(d,e), gt(d) = sum_e u_e lam(d,e) (the transpose of the rank-one coupling), in
// reverse traversal order.  M^T = Vp_T blockdiag Wp_T with Vp_T = Wp^T J, Wp_T = J Vp^T,
// J = diag(+1 for Re and real indices, -1 for Im indices), so the same block solve applies, with the
// coupling vector t (instead of uh) and the trace weights J uh (instead of t).  Templates take ADJ.
//
// Index conventions: a cell array v[e + P*d] holds Legendre degree d in x and e in y (the psi layout);
// a modal array Z[b + P*a] holds packed x-mode a and y-mode b.
#pragma once

#include <cuda_runtime.h>

#include "modal_tables.h"

namespace idc {

template <bool NEG>
__host__ __device__ constexpr double flip_sign(int d) {
    return (NEG && (d & 1)) ? -1.0 : 1.0;
}

// J of the transposed basis: -1 on the Im index of each complex pair.
template <int P>
__host__ __device__ constexpr double jsign(int k) {
    return (k < 2 * ModalTable<P>::kPairs && (k & 1)) ? -1.0 : 1.0;
}
// Trace weight t_k of packed index k: column sums of Vp (1 for a pair's Re index and the real index).
template <int P>
__host__ __device__ constexpr double tweight(int k) {
    return (k < 2 * ModalTable<P>::kPairs && (k & 1)) ? 0.0 : 1.0;
}
// Basis of the forward (ADJ = false) or transposed (ADJ = true) cell operator: packed coefficients
// out = Wb v Wb^T, cell values v = Vb Z Vb^T; coupling vector of the incoming traces and weights of the
// outgoing traces.
template <int P, bool ADJ>
__host__ __device__ constexpr double basis_w(int a, int d) {
    return ADJ ? jsign<P>(a) * ModalTable<P>::V(d, a) : ModalTable<P>::W(a, d);
}
template <int P, bool ADJ>
__host__ __device__ constexpr double basis_v(int d, int a) {
    return ADJ ? ModalTable<P>::W(a, d) * jsign<P>(a) : ModalTable<P>::V(d, a);
}
template <int P, bool ADJ>
__host__ __device__ constexpr double couple_w(int k) {
    return ADJ ? tweight<P>(k) : ModalTable<P>::uh(k);
}
template <int P, bool ADJ>
__host__ __device__ constexpr double trace_w(int k) {
    return ADJ ? jsign<P>(k) * ModalTable<P>::uh(k) : tweight<P>(k);
}

// Per-ordinate constants of the modal cell step (compute type T).
template <int P, typename T>
struct ModalOrdinate {
    T ax, ay;        // |xi|/dx, |eta|/dy
    T cx[P], cy[P];  // ax * uh, ay * uh
    // denominators minus s, per 2-D block (pair x pair: D+ = ax lam + ay conj(lam) + s and
    // D- = ax lam + ay lam + s share the real part; pair x real, real x pair, real x real)
    T pp_re, pp_im_p, pp_im_m, pr_re, pr_im, rp_re, rp_im, rr_re;
};

template <int P, typename T, bool ADJ = false>
__device__ __forceinline__ ModalOrdinate<P, T> modal_ordinate(double axd, double ayd) {
    using Tab = ModalTable<P>;
    ModalOrdinate<P, T> o{};
    o.ax = T(axd);
    o.ay = T(ayd);
#pragma unroll
    for (int k = 0; k < P; ++k) {
        o.cx[k] = T(axd * couple_w<P, ADJ>(k));
        o.cy[k] = T(ayd * couple_w<P, ADJ>(k));
    }
    if constexpr (Tab::kPairs > 0) {
        o.pp_re = T((axd + ayd) * Tab::mu(0));
        o.pp_im_p = T((axd - ayd) * Tab::nu(0));
        o.pp_im_m = T((axd + ayd) * Tab::nu(0));
    }
    if constexpr (Tab::kPairs > 0 && Tab::kHasReal) {
        // explicit fused multiply-adds: every kernel that inlines this rounds these sums the same way
        o.pr_re = T(fma(axd, Tab::mu(0), ayd * Tab::lam_real()));
        o.pr_im = T(axd * Tab::nu(0));
        o.rp_re = T(fma(axd, Tab::lam_real(), ayd * Tab::mu(0)));
        o.rp_im = T(ayd * Tab::nu(0));
    }
    if constexpr (Tab::kHasReal) o.rr_re = T((axd + ayd) * Tab::lam_real());
    return o;
}

// Reciprocal denominators of one cell: complex 1/D as (re, im); the pair x pair block's carry the
// factor 1/2 of its change of basis.
template <int P, typename T>
struct ModalRecip {
    T p_re, p_im, m_re, m_im;   // pair x pair: 1/(2 D+), 1/(2 D-)
    T pr_re, pr_im, rp_re, rp_im, rr;
};

// 1/x for the FP32 solves: the hardware approximation (error below 1 ulp); the FP32 solve is either
// refined in FP64 or accepted at FP32 accuracy.
__device__ __forceinline__ float recip_fast(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Reciprocals of the cell's |D|^2 (positive reals).  FP64: one correctly rounded reciprocal of their
// product and a product chain (Montgomery's simultaneous inversion); the product of the five |D|^2 of
// P = 3 stays finite for |D| below 1e30.  FP32: one hardware reciprocal each.
template <int K>
__device__ __forceinline__ void batch_recip(double (&v)[K]) {
    double pre[K];
    pre[0] = v[0];
#pragma unroll
    for (int k = 1; k < K; ++k) pre[k] = pre[k - 1] * v[k];
    double inv = __drcp_rn(pre[K - 1]);
#pragma unroll
    for (int k = K - 1; k > 0; --k) {
        const double vk = v[k];
        v[k] = inv * pre[k - 1];
        inv *= vk;
    }
    v[0] = inv;
}
template <int K>
__device__ __forceinline__ void batch_recip(float (&v)[K]) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = recip_fast(v[k]);
}

template <int P, typename T>
__device__ __forceinline__ ModalRecip<P, T> modal_recip(const ModalOrdinate<P, T> &o, T s) {
    using Tab = ModalTable<P>;
    ModalRecip<P, T> r{};
    if constexpr (P == 1) {
        T v[1] = {o.rr_re + s};
        batch_recip<1>(v);
        r.rr = v[0];
    } else if constexpr (P == 2) {
        const T re = o.pp_re + s;
        T v[2] = {T(2) * fma(re, re, o.pp_im_p * o.pp_im_p), T(2) * fma(re, re, o.pp_im_m * o.pp_im_m)};
        batch_recip<2>(v);
        r.p_re = re * v[0];
        r.p_im = -o.pp_im_p * v[0];
        r.m_re = re * v[1];
        r.m_im = -o.pp_im_m * v[1];
    } else {
        static_assert(Tab::kPairs == 1 && Tab::kHasReal, "P = 3 layout");
        const T re = o.pp_re + s, a = o.pr_re + s, b = o.rp_re + s, c = o.rr_re + s;
        T v[5] = {T(2) * fma(re, re, o.pp_im_p * o.pp_im_p), T(2) * fma(re, re, o.pp_im_m * o.pp_im_m),
                  fma(a, a, o.pr_im * o.pr_im), fma(b, b, o.rp_im * o.rp_im), c};
        batch_recip<5>(v);
        r.p_re = re * v[0];
        r.p_im = -o.pp_im_p * v[0];
        r.m_re = re * v[1];
        r.m_im = -o.pp_im_m * v[1];
        r.pr_re = a * v[2];
        r.pr_im = -o.pr_im * v[2];
        r.rp_re = b * v[3];
        r.rp_im = -o.rp_im * v[3];
        r.rr = v[4];
    }
    return r;
}

// out(a,b) = sum_{d,e} Wp(a,d) sx^d Wp(b,e) sy^e v(d,e): packed modal coefficients of a (sign-flipped)
// cell array.
template <int P, bool XN, bool YN, typename T, bool ADJ = false>
__device__ __forceinline__ void modal_forward(T (&out)[P * P], const T (&v)[P * P]) {
    T t[P * P];
#pragma unroll
    for (int a = 0; a < P; ++a)
#pragma unroll
        for (int e = 0; e < P; ++e) {
            T acc = v[e] * T(basis_w<P, ADJ>(a, 0));
#pragma unroll
            for (int d = 1; d < P; ++d) acc = fma(T(basis_w<P, ADJ>(a, d) * flip_sign<XN>(d)), v[e + P * d], acc);
            t[e + P * a] = acc;
        }
#pragma unroll
    for (int a = 0; a < P; ++a)
#pragma unroll
        for (int b = 0; b < P; ++b) {
            T acc = t[P * a] * T(basis_w<P, ADJ>(b, 0));
#pragma unroll
            for (int e = 1; e < P; ++e) acc = fma(T(basis_w<P, ADJ>(b, e) * flip_sign<YN>(e)), t[e + P * a], acc);
            out[b + P * a] = acc;
        }
}

// v(d,e) = sx^d sy^e sum_{a,b} Vp(d,a) Vp(e,b) Z(a,b): the cell array (unflipped) of modal coefficients.
template <int P, bool XN, bool YN, typename T, bool ADJ = false>
__device__ __forceinline__ void modal_backward(T (&v)[P * P], const T (&Z)[P * P]) {
    T t[P * P];   // t(d, b) = sx^d sum_a Vb(d,a) Z(a,b)
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int b = 0; b < P; ++b) {
            T acc = Z[b] * T(basis_v<P, ADJ>(d, 0) * flip_sign<XN>(d));
#pragma unroll
            for (int a = 1; a < P; ++a) acc = fma(T(basis_v<P, ADJ>(d, a) * flip_sign<XN>(d)), Z[b + P * a], acc);
            t[b + P * d] = acc;
        }
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e) {
            T acc = t[P * d] * T(basis_v<P, ADJ>(e, 0) * flip_sign<YN>(e));
#pragma unroll
            for (int b = 1; b < P; ++b) acc = fma(T(basis_v<P, ADJ>(e, b) * flip_sign<YN>(e)), t[b + P * d], acc);
            v[e + P * d] = acc;
        }
}

// Z = blocks^-1 Y in place.
template <int P, typename T>
__device__ __forceinline__ void modal_block_solve(T (&Y)[P * P], const ModalRecip<P, T> &r) {
    using Tab = ModalTable<P>;
    if constexpr (Tab::kPairs > 0) {
        // pair x pair: (rr, ri, ir, ii) -> z+ = (rr + ii) + i(ir - ri), z- = (rr - ii) + i(ir + ri)
        const T rr = Y[0], ri = Y[1], ir = Y[P], ii = Y[P + 1];
        const T zp_re = rr + ii, zp_im = ir - ri, zm_re = rr - ii, zm_im = ir + ri;
        const T ap_re = fma(zp_re, r.p_re, -zp_im * r.p_im), ap_im = fma(zp_re, r.p_im, zp_im * r.p_re);
        const T am_re = fma(zm_re, r.m_re, -zm_im * r.m_im), am_im = fma(zm_re, r.m_im, zm_im * r.m_re);
        Y[0] = ap_re + am_re;       // rr = Re(z+ + z-)
        Y[P] = ap_im + am_im;       // ir = Im(z+ + z-)
        Y[1] = am_im - ap_im;       // ri = -Im(z+ - z-)
        Y[P + 1] = ap_re - am_re;   // ii = Re(z+ - z-)
    }
    if constexpr (Tab::kPairs > 0 && Tab::kHasReal) {
        // pair x real: (Y(0,2), Y(1,2)) complex; real x pair: (Y(2,0), Y(2,1)) complex
        const T a_re = Y[2], a_im = Y[2 + P];
        Y[2] = fma(a_re, r.pr_re, -a_im * r.pr_im);
        Y[2 + P] = fma(a_re, r.pr_im, a_im * r.pr_re);
        const T b_re = Y[2 * P], b_im = Y[2 * P + 1];
        Y[2 * P] = fma(b_re, r.rp_re, -b_im * r.rp_im);
        Y[2 * P + 1] = fma(b_re, r.rp_im, b_im * r.rp_re);
    }
    if constexpr (Tab::kHasReal) Y[P * P - 1] *= r.rr;
}

// Sum of v[k] * w(k) over k with compile-time weights (zero weights skipped, unit weights added).
template <int P, typename T, typename W>
__device__ __forceinline__ T weighted_sum(const T *v, int stride, W w) {
    T acc = T(0);
    bool first = true;
#pragma unroll
    for (int k = 0; k < P; ++k) {
        const double c = w(k);
        if (c == 0.0) continue;
        const T term = v[k * stride];
        if (first)
            acc = (c == 1.0) ? term : T(c) * term;
        else
            acc = (c == 1.0) ? acc + term : fma(T(c), term, acc);
        first = false;
    }
    return acc;
}

// One modal cell step: Z from the cell's packed source S, the incoming packed traces fh (x-upwind cell)
// and gh (y-upwind cell); then fh <- outgoing x trace, gh_out <- outgoing y trace.  Coupling terms with
// a zero coupling weight are skipped at compile time.
template <int P, typename T, bool ADJ = false>
__device__ __forceinline__ void modal_step(T (&Z)[P * P], const T (&S)[P * P], T (&fh)[P], const T (&gh)[P],
                                           T (&gh_out)[P], const ModalOrdinate<P, T> &o, const ModalRecip<P, T> &r) {
#pragma unroll
    for (int a = 0; a < P; ++a)
#pragma unroll
        for (int b = 0; b < P; ++b) {
            T z = S[b + P * a];
            if (couple_w<P, ADJ>(b) != 0.0) z = fma(o.cy[b], gh[a], z);
            if (couple_w<P, ADJ>(a) != 0.0) z = fma(o.cx[a], fh[b], z);
            Z[b + P * a] = z;
        }
    modal_block_solve<P, T>(Z, r);
#pragma unroll
    for (int b = 0; b < P; ++b) fh[b] = weighted_sum<P, T>(Z + b, P, [](int k) { return trace_w<P, ADJ>(k); });
#pragma unroll
    for (int a = 0; a < P; ++a) gh_out[a] = weighted_sum<P, T>(Z + P * a, 1, [](int k) { return trace_w<P, ADJ>(k); });
}

// Physical-basis solve x = A'^-1 B (flipped, scaled frame) through the modal basis, in type T.
template <int P, typename T, bool ADJ = false>
__device__ __forceinline__ void modal_solve_phys(T (&x)[P * P], const T (&B)[P * P], const ModalRecip<P, T> &r) {
    T Z[P * P];
    modal_forward<P, false, false, T, ADJ>(Z, B);
    modal_block_solve<P, T>(Z, r);
    modal_backward<P, false, false, T, ADJ>(x, Z);
}

// Entry (d, a) of the 1-D upwind matrix M (xi > 0): (2d+1)(1 - 2[a < d, d - a odd]).
__host__ __device__ constexpr double upwind_m(int d, int a) {
    return (a < d && ((d - a) & 1)) ? -double(2 * d + 1) : double(2 * d + 1);
}

// r = B - A' x in FP64, A' = ax (M (x) I) + ay (I (x) M) + s I, or its transpose (ADJ).
template <int P, bool ADJ = false>
__device__ __forceinline__ void phys_residual(double (&res)[P * P], const double (&B)[P * P], const double (&x)[P * P],
                                              double ax, double ay, double s) {
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e) {
            double mx = 0.0, my = 0.0;
#pragma unroll
            for (int a = 0; a < P; ++a) mx = fma(ADJ ? upwind_m(a, d) : upwind_m(d, a), x[e + P * a], mx);
#pragma unroll
            for (int b = 0; b < P; ++b) my = fma(ADJ ? upwind_m(b, e) : upwind_m(e, b), x[b + P * d], my);
            res[e + P * d] = B[e + P * d] - fma(ax, mx, fma(ay, my, s * x[e + P * d]));
        }
}

}  // namespace idc
