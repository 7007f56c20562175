// Fused local systems of the NNGP fit step and predict on B200 (sm_100a).
//
// For every point p with neighbours nbr[p, 0..m-1] (reference: Nngpr._log_likelihood_worker,
// base_nngpr.py:538-614, and Nngpr._predict_worker, :1032-1135) one kernel does, without
// writing any m x m matrix to HBM:
//   fill     K of the augmented system [neighbours..., p] for
//            rbf_level * exp(-|dx / l|^2 / 2) + const (+ noise + alpha on the diagonal), a -1
//            neighbour giving an identity row/column (fill_nn_kernel semantics,
//            cuda_kernel_accelerators.py:748-863);
//   factor   the Cholesky factor of the augmented matrix with p LAST: its last row is
//            l = L_nn^-1 k and its last pivot is sigma^2 = K_pp - k^T K_nn^-1 k;
//   solve    z_c = L_nn^-1 y_nn,c, mu_c = l . z_c, r_c = y_c - mu_c;
//   reduce   log-likelihood -r^2 / (2 sigma^2) - log sigma - log(2 pi) / 2 summed in FP64
//            (base_nngpr.py:578-584), or mean/variance for predict (:1117-1127);
//   adjoint  (gradient) b = K_nn^-1 k and v = sum_c (r_c / sigma^2) K_nn^-1 y_nn,c by two
//            backward solves, then d loglik / d theta_t = sum_ij G_ij dK_ij/dtheta_t with
//            G_pp = w, G_pj = v_j / 2 - w b_j, G_jk = w b_j b_k - (b_j v_k + v_j b_k) / 2,
//            w = sum_c (r_c^2 / sigma^2 - 1) / (2 sigma^2): algebraically the reference's
//            gradient (base_nngpr.py:586-614), evaluated by recomputing the fill instead of
//            storing dK (n m^2 n_theta values in the reference).
//
// Two kernels:
//   * warp kernel (m <= 32): one warp per point, lane i owns row i of the factor in registers;
//     FP32 with an FP64 re-solve of the system when a pivot is below the threshold (or FP64
//     throughout for double inputs);
//   * block kernel (32 < m <= ~150): one CTA per point, the augmented matrix in shared memory,
//     FP64.
// Per-point terms are summed in FP64: per warp, per CTA, then in fixed order by a finalize
// kernel (deterministic for a given launch shape).
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <type_traits>

#include "common.cuh"

namespace nngp {

constexpr int kMaxDimLocal = 256;
constexpr int kMaxTheta = kMaxDimLocal + 3;
constexpr int kWarpM = 32;
constexpr int kLocWarps = 4;
constexpr double kHalfLog2Pi = 0.91893853320467274178;

struct LocalArgs {
    double rbf, cst, noise, alpha;
    double pivot_abs;  // FP32 systems with a pivot below this are re-solved in FP64
    int64_t n_rows;    // rows of x_ref / y_ref (neighbour index bound)
    int64_t n_points;
    int d, ydim, m;
    int ard;  // 1: per-feature length scales
    int family;  // stationary part: NNGP_FAMILY_RBF or a Matern (include/nngp_b200.h)
    int64_t alpha_below;  // alpha goes on the diagonal slots of neighbours with index < alpha_below
    int weights_out;      // predict: write w = K_nn^-1 k (a.m per point) to `mean` instead of the mean
    int idx_rbf, idx_const, idx_noise, idx_ls, n_theta;
    unsigned long long *fp64_count;  // systems re-solved in FP64 are added here (may be null)
    // fit step with FP32 inputs: bit p marks point p (counted from the launch's first row), whose
    // FP32 system needs the FP64 re-solve that local_redo_kernel then runs (predict re-solves in
    // place and leaves this null)
    uint32_t *redo_bits;
    // device block of nngp_theta_params (may be null): [rbf, cst, noise, pivot_abs, 1/l_f ...];
    // when set, the kernels take these values instead of the fields above
    const double *dev_params;
    double inv_ls[kMaxDimLocal];
};

// The hyperparameter values a kernel works with: from the arguments, or from the device block
// of a theta that never left the device.
struct Hyp {
    double rbf, cst, noise, pivot_abs;
    const double *inv_ls;
};
__device__ __forceinline__ Hyp hyp_of(const LocalArgs &a) {
    if (a.dev_params) {
        const double *q = a.dev_params;
        return Hyp{q[0], q[1], q[2], q[3], q + 4};
    }
    return Hyp{a.rbf, a.cst, a.noise, a.pivot_abs, a.inv_ls};
}

template <typename T> __device__ __forceinline__ T dsqrt(T v) { return sqrt(v); }
template <typename T> __device__ __forceinline__ T drsqrt(T v) { return rsqrt(v); }
template <> __device__ __forceinline__ float drsqrt<float>(float v) { return rsqrtf(v); }
template <typename T> __device__ __forceinline__ T dexp(T v) { return exp(v); }
template <> __device__ __forceinline__ float dexp<float>(float v) { return expf(v); }

// Unit-amplitude stationary part s of the kernel at squared scaled distance sq (formulas of
// nngpr/batched_kernels.py:1070-1088 for the Matern kernels; RBF exp(-sq / 2)).
template <bool MATERN, typename T> __device__ __forceinline__ T kern_s(int family, T sq) {
    if (!MATERN || family == NNGP_FAMILY_RBF) return dexp<T>(T(-0.5) * sq);
    if (family == NNGP_FAMILY_MATERN12) return dexp<T>(-dsqrt<T>(sq));
    if (family == NNGP_FAMILY_MATERN32) {
        const T r = dsqrt<T>(T(3) * sq);
        return (T(1) + r) * dexp<T>(-r);
    }
    const T r = dsqrt<T>(T(5) * sq);
    return (T(1) + r + r * r / T(3)) * dexp<T>(-r);
}

// g with d s / d log l_f = g * t_f^2 (t_f the scaled difference of feature f); isotropic:
// d s / d log l = g * sq.  `s` is kern_s at the same sq.  Reference gradients:
// nngpr/batched_kernels.py:1108-1120 (Matern), :895-898 (RBF).
template <bool MATERN, typename T> __device__ __forceinline__ T kern_g(int family, T sq, T s) {
    if (!MATERN || family == NNGP_FAMILY_RBF) return s;
    if (family == NNGP_FAMILY_MATERN12) {
        const T r = dsqrt<T>(sq);
        return r > T(0) ? s / r : T(0);  // every t_f is 0 where r is
    }
    if (family == NNGP_FAMILY_MATERN32) return T(3) * dexp<T>(-dsqrt<T>(T(3) * sq));
    const T r = dsqrt<T>(T(5) * sq);
    return T(5) / T(3) * (T(1) + r) * dexp<T>(-r);
}

// ---------------------------------------------------------------------------------------
// Warp kernel
// ---------------------------------------------------------------------------------------
// Shared memory per warp (bytes): two Cholesky column slots 2 x kWarpM doubles (16-byte
// aligned, first) | xs (kWarpM + 1) x ds doubles | P kWarpM x (kWarpM + 1) doubles | inverse
// diagonal kWarpM doubles | gradient accumulator n_theta doubles.  P holds two triangles: the
// strictly lower part of the factor, L[i][k] at P[i][k] (k < i), and the fill's kernel values
// of the lower triangle, E[i][k] at P[k][i + 1] (k <= i, so column i + 1 > row k), which the
// gradient reuses instead of recomputing them.  One array for both halves the footprint of a
// warp (more resident warps per SM).
struct WarpSmem {
    int ds;  // row stride of xs (d + 1; FP32 systems use whole float4s, see warp_system)
    size_t c_bytes, xs_bytes, l_bytes, idg_bytes, g_bytes, r_bytes, total;
    size_t xs_off, l_off, idg_off, g_off, r_off;
    // f32: FP32 inputs, whose systems also keep the fill's squared distances (kWarpM x (kWarpM + 1)
    // floats) for the gradient instead of recomputing them
    // sys4: the warp only ever solves FP32 systems (the fit step's FP32 kernel), so the column
    // slots, xs, P and the inverse diagonal take 4-byte elements
    __host__ __device__ static WarpSmem make(int d, int n_theta, bool f32 = false, bool sys4 = false) {
        WarpSmem s;
        const size_t e = sys4 ? 4 : 8;
        s.ds = d + 1;
        s.c_bytes = (size_t)2 * kWarpM * e;
        s.xs_bytes = sys4 ? (size_t)(kWarpM + 1) * 4 * (((d + 3) / 4) | 1) * 4 : (size_t)(kWarpM + 1) * s.ds * 8;
        s.l_bytes = (size_t)kWarpM * (kWarpM + 1) * e;
        s.idg_bytes = (size_t)kWarpM * e;
        s.g_bytes = (size_t)(n_theta > 0 ? n_theta : 1) * 8;
        s.xs_off = s.c_bytes;
        s.l_off = s.xs_off + s.xs_bytes;
        s.idg_off = s.l_off + s.l_bytes;
        s.g_off = s.idg_off + s.idg_bytes;
        s.r_bytes = f32 ? (size_t)kWarpM * (kWarpM + 1) * 4 : 0;
        s.r_off = s.g_off + s.g_bytes;
        s.total = (s.r_off + s.r_bytes + 15) / 16 * 16;
        return s;
    }
};

// Vector of VW elements of TC read with one 16-byte shared-memory load.
template <typename TC> struct Vec16;
template <> struct Vec16<double> {
    static constexpr int VW = 2;
    using T = double2;
    __device__ static double get(const double2 &v, int e) { return e == 0 ? v.x : v.y; }
};
template <> struct Vec16<float> {
    static constexpr int VW = 4;
    using T = float4;
    __device__ static float get(const float4 &v, int e) { return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w)); }
};

// Solves point p's system in precision TC.  Returns false (and commits nothing) when TC is
// float and a pivot fell below the FP64 threshold.
template <typename TC, typename TIn, bool GRAD, bool PRED, bool MATERN>
__device__ __forceinline__ bool warp_system(const LocalArgs &a, int64_t p, int lane, const TIn *__restrict__ x_ref,
                                            const TIn *__restrict__ y_ref, const TIn *__restrict__ x_pt,
                                            const TIn *__restrict__ y_pt, const int32_t *__restrict__ nbr,
                                            unsigned char *wsm, double &ll_acc, TIn *__restrict__ mean,
                                            TIn *__restrict__ var, int32_t *__restrict__ flags) {
    constexpr int M = kWarpM;
    const Hyp h = hyp_of(a);
    const unsigned FULL = 0xffffffffu;
    const WarpSmem lay = WarpSmem::make(a.d, a.n_theta, std::is_same<TIn, float>::value,
                                        std::is_same<TIn, float>::value && !PRED && std::is_same<TC, float>::value);
    TC *colbuf = reinterpret_cast<TC *>(wsm);  // two column slots of kWarpM, 16-byte aligned
    TC *xs = reinterpret_cast<TC *>(wsm + lay.xs_off);
    TC *Ls = reinterpret_cast<TC *>(wsm + lay.l_off);
    TC *idg = reinterpret_cast<TC *>(wsm + lay.idg_off);
    double *gacc = reinterpret_cast<double *>(wsm + lay.g_off);
    constexpr bool STASH = GRAD && !MATERN;  // RBF gradient: reuse the fill's exponentials
    // FP32 RBF systems also keep the squared distances (the gradient's only other use of the fill)
    constexpr bool STASH_R = STASH && std::is_same<TC, float>::value && std::is_same<TIn, float>::value;
    float *Rs = reinterpret_cast<float *>(wsm + lay.r_off);
    // FP32 rows of xs are whole float4s, an odd number of them (one 16-byte load per 4 features,
    // rows of different lanes in distinct bank groups), zero padded: the padding adds (0 - 0)^2
    // terms, so every sum is the same as over the d features alone
    constexpr bool VEC4 = std::is_same<TC, float>::value;
    const int d = a.d;
    const int ds = VEC4 ? 4 * (((d + 3) / 4) | 1) : lay.ds;

    // ---- neighbour of this lane --------------------------------------------------------
    int32_t j = -1;
    if (lane < a.m) {
        j = __ldg(nbr + p * a.m + lane);
        if (j < -1 || (int64_t)j >= a.n_rows) {
            flag_or(flags, NNGP_FLAG_BAD_INDEX);
            j = -1;
        }
    }
    const bool valid = j >= 0;
    const unsigned vmask = __ballot_sync(FULL, valid);

    // ---- gather scaled coordinates: rows 0..M-1 neighbours, row M the point ------------
    __syncwarp();
    for (int f = 0; f < d; ++f) {
        const TC s = (TC)h.inv_ls[a.ard ? f : 0];
        xs[lane * ds + f] = valid ? (TC)x_ref[(int64_t)j * d + f] * s : TC(0);
    }
    for (int f = lane; f < d; f += 32) xs[M * ds + f] = (TC)x_pt[p * d + f] * (TC)h.inv_ls[a.ard ? f : 0];
    if (VEC4) {
        for (int f = d; f < ds; ++f) xs[lane * ds + f] = TC(0);
        for (int f = d + lane; f < ds; f += 32) xs[M * ds + f] = TC(0);
    }
    __syncwarp();

    // ---- fill: squared scaled distances, then kernel values ------------------------------
    TC r[M];
    TC rp = TC(0);
#pragma unroll
    for (int k = 0; k < M; ++k) r[k] = TC(0);
    if constexpr (VEC4) {
        const float4 *xs4 = reinterpret_cast<const float4 *>(xs);
        const int ds4 = ds / 4, nf4 = (d + 3) / 4;
        for (int f4 = 0; f4 < nf4; ++f4) {
            const float4 xi = xs4[lane * ds4 + f4];
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const float4 xk = xs4[k * ds4 + f4];
                float t = xi.x - xk.x;
                r[k] = fmaf(t, t, r[k]);
                t = xi.y - xk.y;
                r[k] = fmaf(t, t, r[k]);
                t = xi.z - xk.z;
                r[k] = fmaf(t, t, r[k]);
                t = xi.w - xk.w;
                r[k] = fmaf(t, t, r[k]);
            }
            const float4 xp = xs4[M * ds4 + f4];
            float t = xi.x - xp.x;
            rp = fmaf(t, t, rp);
            t = xi.y - xp.y;
            rp = fmaf(t, t, rp);
            t = xi.z - xp.z;
            rp = fmaf(t, t, rp);
            t = xi.w - xp.w;
            rp = fmaf(t, t, rp);
        }
    } else {
        for (int f = 0; f < d; ++f) {
            const TC xi = xs[lane * ds + f];
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const TC t = xi - xs[k * ds + f];
                r[k] = fma(t, t, r[k]);
            }
            const TC t = xi - xs[M * ds + f];
            rp = fma(t, t, rp);
        }
    }
    const TC rbf = (TC)h.rbf, cst = (TC)h.cst;
    const TC diag_add = (TC)h.noise + ((int64_t)j < a.alpha_below ? (TC)a.alpha : TC(0));
#pragma unroll
    for (int k = 0; k < M; ++k) {
        const bool vk = (vmask >> k) & 1u;
        const TC e = rbf * kern_s<MATERN>(a.family, r[k]);
        if (STASH && k <= lane) Ls[k * (M + 1) + lane + 1] = e;  // E[lane][k], upper triangle of P
        if (STASH_R) Rs[lane * (M + 1) + k] = (float)r[k];
        TC kv = (valid && vk) ? e + cst : TC(0);
        if (k == lane) kv = valid ? kv + diag_add : TC(1);
        r[k] = kv;
    }
    const TC ep0 = rbf * kern_s<MATERN>(a.family, rp);  // kept for the gradient
    TC kvec = valid ? ep0 + cst : TC(0);                 // K[p][lane]
    const TC kpp = rbf + cst + (TC)h.noise + (PRED ? TC(0) : (TC)a.alpha);

    // ---- Cholesky of the neighbour block fused with l = L^-1 k ----------------------------
    // A lane's own results (its pivot's reciprocal, l_lane, z_lane, b_lane, v_lane) are not picked
    // out of the step that produces them: the running value a lane holds stops changing once
    // its own step is reached, so each is formed once after the loop, from the same operands.
    TC minpiv = TC(3.0e38);
    TC ss = TC(0);
#pragma unroll
    for (int k = 0; k < M; ++k) {
        const TC piv = __shfl_sync(FULL, r[k], k);
        minpiv = fmin(minpiv, piv);
        const TC inv = drsqrt<TC>(piv);  // 1 / L_kk
        r[k] = r[k] * inv;               // L_jk, and L_kk = piv * inv on lane k itself
        if (lane == k) idg[k] = inv;
        const TC lk = __shfl_sync(FULL, kvec, k) * inv;
        if (lane > k) kvec = fma(-r[k], lk, kvec);
        ss = fma(lk, lk, ss);
        if (k + 1 < M) {
            // column k of L to a shared slot (alternating slots: a lane that wrote column k has
            // finished reading column k - 1), then every lane reads L[jj][k], jj > k, as
            // broadcast 16-byte loads instead of one shuffle per element
            TC *col = colbuf + (k & 1) * M;
            col[lane] = r[k];
            __syncwarp();
            using V = Vec16<TC>;
            const typename V::T *cv = reinterpret_cast<const typename V::T *>(col);
#pragma unroll
            for (int q = (k + 1) / V::VW; q < M / V::VW; ++q) {
                const typename V::T v = cv[q];
#pragma unroll
                for (int e = 0; e < V::VW; ++e) {
                    const int jj = q * V::VW + e;
                    if (jj > k) r[jj] = fma(-r[k], V::get(v, e), r[jj]);
                }
            }
        }
    }
    const TC s2 = kpp - ss;
    if constexpr (std::is_same<TC, float>::value) {
        if (!(minpiv >= (TC)h.pivot_abs) || !(s2 >= (TC)h.pivot_abs)) return false;  // NaN-safe
    }
    if (!(minpiv > TC(0)) || !(s2 > TC(0))) flag_or(flags, NNGP_FLAG_NOT_PD);

    // L (strictly lower part, the upper part of P keeps E) and inverse diagonal to shared
    // memory for the backward solves
#pragma unroll
    for (int k = 0; k < M; ++k)
        if (k < lane) Ls[lane * (M + 1) + k] = r[k];
    const TC l_own = kvec * idg[lane];  // l_lane (this lane's own write of idg)
    __syncwarp();

    if (PRED && a.weights_out) {
        // conditioning weights w = L^-T l = K_nn^-1 k and the variance term s2 (no outputs yet:
        // the full-conditioning recursion combines them with earlier predictions)
        TC bv = l_own;
#pragma unroll
        for (int k = M - 1; k >= 0; --k) {
            const TC bk = __shfl_sync(FULL, bv, k) * idg[k];
            const TC lkj = Ls[k * (M + 1) + lane];
            if (lane < k) bv = fma(-lkj, bk, bv);
        }
        const TC b_own = bv * idg[lane];
        if (lane < a.m) mean[p * a.m + lane] = (TIn)b_own;
        if (lane == 0) var[p] = (TIn)s2;
        return true;
    }

    // ---- outputs ------------------------------------------------------------------------
    TC zw = TC(0);
    TC wsum = TC(0);
    double ll = 0.0;
    for (int c = 0; c < a.ydim; ++c) {
        TC yv = valid ? (TC)y_ref[(int64_t)j * a.ydim + c] : TC(0);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            const TC zk = __shfl_sync(FULL, yv, k) * idg[k];
            if (lane > k) yv = fma(-r[k], zk, yv);
        }
        const TC z_own = yv * idg[lane];
        const TC mu = warp_sum(l_own * z_own);
        if (PRED) {
            if (lane == 0) mean[p * a.ydim + c] = (TIn)mu;
        } else {
            const TC res = (TC)y_pt[p * a.ydim + c] - mu;
            const double rd = (double)res, sd = (double)s2;
            ll += -0.5 * rd * rd / sd - 0.5 * log(sd) - kHalfLog2Pi;
            if (GRAD) {
                const TC rs = res / s2;
                zw = fma(rs, z_own, zw);
                wsum += (res * rs - TC(1)) / (TC(2) * s2);
            }
        }
    }
    if (PRED) {
        if (lane == 0) var[p] = (TIn)s2;
        return true;
    }
    if (!GRAD) {
        if (lane == 0) ll_acc += ll;
        return true;
    }

    // ---- adjoint: b = L^-T l, v = L^-T zw ------------------------------------------------
    TC bv = l_own, vv = zw;
#pragma unroll
    for (int k = M - 1; k >= 0; --k) {
        const TC ik = idg[k];
        const TC bk = __shfl_sync(FULL, bv, k) * ik;
        const TC vk = __shfl_sync(FULL, vv, k) * ik;
        const TC lkj = Ls[k * (M + 1) + lane];
        if (lane < k) {
            bv = fma(-lkj, bk, bv);
            vv = fma(-lkj, vk, vv);
        }
    }
    const TC b_own = bv * idg[lane], v_own = vv * idg[lane];

    // the fill's squared distances: kept (FP32 RBF), else recomputed (xs is intact); rp still
    // holds the fill's distance to the point itself
    if constexpr (STASH_R) {
#pragma unroll
        for (int k = 0; k < M; ++k) r[k] = (TC)Rs[lane * (M + 1) + k];
    } else {
#pragma unroll
        for (int k = 0; k < M; ++k) r[k] = TC(0);
        rp = TC(0);
        for (int f = 0; f < d; ++f) {
            const TC xi = xs[lane * ds + f];
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const TC t = xi - xs[k * ds + f];
                r[k] = fma(t, t, r[k]);
            }
            const TC t = xi - xs[M * ds + f];
            rp = fma(t, t, rp);
        }
    }
    TC g_amp = TC(0), g_cst = TC(0), g_noise = TC(0), g_iso = TC(0);
#pragma unroll
    for (int k = 0; k < M; ++k) {
        const TC bk = __shfl_sync(FULL, b_own, k);
        const TC vk = __shfl_sync(FULL, v_own, k);
        const bool vk_ok = (vmask >> k) & 1u;
        const TC G = wsum * b_own * bk - TC(0.5) * (b_own * vk + v_own * bk);
        const TC wgt = (valid && vk_ok) ? (k < lane ? TC(2) : (k == lane ? TC(1) : TC(0))) : TC(0);
        const TC s = STASH ? TC(0) : kern_s<MATERN>(a.family, r[k]);
        const TC gw = wgt * G;
        // E[lane][k] for k <= lane (wgt is 0 above the diagonal, where P holds L)
        const TC ge = gw * (STASH ? (k <= lane ? Ls[k * (M + 1) + lane + 1] : TC(0)) : rbf * s);
        const TC gl = MATERN ? gw * (rbf * kern_g<MATERN>(a.family, r[k], s)) : ge;
        g_amp += ge;
        g_cst += gw;
        g_iso = fma(gl, r[k], g_iso);
        if (k == lane && valid) g_noise += G;
        r[k] = gl;  // kept for the per-feature length-scale terms
    }
    // pair (p, lane), weight 2, and (p, p)
    const TC Gp = valid ? TC(0.5) * v_own - wsum * b_own : TC(0);
    const TC sp = MATERN ? kern_s<MATERN>(a.family, rp) : TC(0);
    const TC gpe = TC(2) * Gp * (MATERN ? rbf * sp : ep0);
    const TC gpl = MATERN ? TC(2) * Gp * (rbf * kern_g<MATERN>(a.family, rp, sp)) : gpe;
    g_amp += gpe;
    g_cst += TC(2) * Gp;
    g_iso = fma(gpl, rp, g_iso);
    const double amp_t = (double)warp_sum(g_amp) + (double)wsum * h.rbf;
    const double cst_t = (double)warp_sum(g_cst) + (double)wsum;
    const double noi_t = (double)warp_sum(g_noise) + (double)wsum;
    const double iso_t = (double)warp_sum(g_iso);
    if (lane == 0) {
        ll_acc += ll;
        if (a.idx_rbf >= 0) gacc[a.idx_rbf] += amp_t;
        if (a.idx_const >= 0) gacc[a.idx_const] += h.cst * cst_t;
        if (a.idx_noise >= 0) gacc[a.idx_noise] += h.noise * noi_t;
        if (a.idx_ls >= 0 && !a.ard) gacc[a.idx_ls] += iso_t;
    }
    if (a.idx_ls >= 0 && a.ard) {
        for (int f = 0; f < d; ++f) {
            const TC xi = xs[lane * ds + f];
            TC acc = TC(0);
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const TC t = xi - xs[k * ds + f];
                acc = fma(r[k] * t, t, acc);
            }
            const TC t = xi - xs[M * ds + f];
            acc = fma(gpl * t, t, acc);
            const double s = (double)warp_sum(acc);
            if (lane == 0) gacc[a.idx_ls + f] += s;
        }
    }
    __syncwarp();
    return true;
}

// Resident CTAs per SM the register budget is set for: the fit step's FP32 kernel (FP32 systems
// only, 4-byte warp layout) 4, the others 3.
template <typename TIn, bool PRED> constexpr int kLocMinBlocks = (std::is_same<TIn, float>::value && !PRED) ? 4 : 3;

template <typename TIn, bool GRAD, bool PRED, bool MATERN>
__global__ void __launch_bounds__(kLocWarps * 32, (kLocMinBlocks<TIn, PRED>)) local_warp_kernel(
    const __grid_constant__ LocalArgs a, const TIn *__restrict__ x_ref, const TIn *__restrict__ y_ref,
    const TIn *__restrict__ x_pt, const TIn *__restrict__ y_pt, const int32_t *__restrict__ nbr,
    double *__restrict__ block_out, TIn *__restrict__ mean, TIn *__restrict__ var, int32_t *__restrict__ flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const WarpSmem lay = WarpSmem::make(a.d, a.n_theta, std::is_same<TIn, float>::value,
                                        std::is_same<TIn, float>::value && !PRED);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wsm = smem_raw + warp * lay.total;
    double *gacc = reinterpret_cast<double *>(wsm + lay.g_off);
    for (int t = lane; t < a.n_theta; t += 32) gacc[t] = 0.0;
    __syncwarp();
    double ll_acc = 0.0;
    bool used_fp64 = false;
    unsigned long long n_fp64 = 0;
    const int64_t nwarps = (int64_t)gridDim.x * kLocWarps;
    for (int64_t p = (int64_t)blockIdx.x * kLocWarps + warp; p < a.n_points; p += nwarps) {
        bool done = false;
        if constexpr (std::is_same<TIn, float>::value) {
            done = warp_system<float, TIn, GRAD, PRED, MATERN>(a, p, lane, x_ref, y_ref, x_pt, y_pt, nbr, wsm, ll_acc, mean,
                                                       var, flags);
        }
        if (!done) {
            if constexpr (std::is_same<TIn, float>::value) {
                used_fp64 = true;
                ++n_fp64;
            }
            if constexpr (std::is_same<TIn, float>::value && !PRED) {
                // the fit step's FP32 kernel carries no FP64 system (registers): the point is
                // marked for local_redo_kernel
                if (lane == 0) atomicOr(a.redo_bits + (p >> 5), 1u << (p & 31));
            } else {
                warp_system<double, TIn, GRAD, PRED, MATERN>(a, p, lane, x_ref, y_ref, x_pt, y_pt, nbr, wsm, ll_acc, mean,
                                                             var, flags);
            }
        }
    }
    if (used_fp64 && lane == 0) {
        flag_or(flags, NNGP_FLAG_FP64_FALLBACK);
        if (a.fp64_count) atomicAdd(a.fp64_count, n_fp64);
    }
    if (PRED) return;
    // CTA reduction in fixed order: warp w's totals -> slot w, then warp 0 sums
    __shared__ double red[kLocWarps];
    if (lane == 0) red[warp] = ll_acc;
    __syncthreads();
    const int nt = 1 + (GRAD ? a.n_theta : 0);
    double *o = block_out + (int64_t)blockIdx.x * nt;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kLocWarps; ++w) s += red[w];
        o[0] = s;
    }
    if (GRAD) {
        for (int t = threadIdx.x; t < a.n_theta; t += blockDim.x) {
            double s = 0.0;
            for (int w = 0; w < kLocWarps; ++w)
                s += reinterpret_cast<const double *>(smem_raw + w * lay.total + lay.g_off)[t];
            o[1 + t] = s;
        }
    }
}

// FP64 re-solve of the fit-step systems the FP32 kernel marked (warp per point, the same warp
// layout); the points of a 32-point word go to one warp, words to warps in a fixed order, so the
// per-CTA partials are deterministic for a given launch shape.
template <bool GRAD, bool MATERN>
__global__ void __launch_bounds__(kLocWarps * 32, 3) local_redo_kernel(
    const __grid_constant__ LocalArgs a, const float *__restrict__ x_ref, const float *__restrict__ y_ref,
    const float *__restrict__ x_pt, const float *__restrict__ y_pt, const int32_t *__restrict__ nbr,
    double *__restrict__ block_out, int32_t *__restrict__ flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const WarpSmem lay = WarpSmem::make(a.d, a.n_theta, true);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wsm = smem_raw + warp * lay.total;
    double *gacc = reinterpret_cast<double *>(wsm + lay.g_off);
    for (int t = lane; t < a.n_theta; t += 32) gacc[t] = 0.0;
    __syncwarp();
    double ll_acc = 0.0;
    const int64_t words = (a.n_points + 31) / 32;
    const int64_t nwarps = (int64_t)gridDim.x * kLocWarps;
    for (int64_t w = (int64_t)blockIdx.x * kLocWarps + warp; w < words; w += nwarps) {
        uint32_t bits = a.redo_bits[w];
        while (bits) {
            const int64_t p = w * 32 + (__ffs(bits) - 1);
            bits &= bits - 1;
            warp_system<double, float, GRAD, false, MATERN>(a, p, lane, x_ref, y_ref, x_pt, y_pt, nbr, wsm, ll_acc,
                                                            nullptr, nullptr, flags);
        }
    }
    __shared__ double red[kLocWarps];
    if (lane == 0) red[warp] = ll_acc;
    __syncthreads();
    const int nt = 1 + (GRAD ? a.n_theta : 0);
    double *o = block_out + (int64_t)blockIdx.x * nt;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kLocWarps; ++w) s += red[w];
        o[0] = s;
    }
    if (GRAD) {
        for (int t = threadIdx.x; t < a.n_theta; t += blockDim.x) {
            double s = 0.0;
            for (int w = 0; w < kLocWarps; ++w)
                s += reinterpret_cast<const double *>(smem_raw + w * lay.total + lay.g_off)[t];
            o[1 + t] = s;
        }
    }
}

// ---------------------------------------------------------------------------------------
// Block kernel (32 < m): one CTA per point, FP64, augmented matrix in shared memory
// ---------------------------------------------------------------------------------------
constexpr int kBlkThreads = 256;

struct BlockSmem {
    int n1, lda, ds;
    size_t a_off, xs_off, vec_off, idx_off, total;
    __host__ __device__ static BlockSmem make(int m, int d) {
        BlockSmem s;
        s.n1 = m + 1;
        s.lda = m + 2;
        s.ds = d;
        size_t off = 0;
        s.a_off = off;
        off += (size_t)s.n1 * s.lda * 8;
        s.xs_off = off;
        off += (size_t)s.n1 * d * 8;
        s.vec_off = off;
        off += (size_t)6 * s.n1 * 8 + 64 * 8;  // yv, z, zw, b, v, tmp + reduction scratch
        s.idx_off = off;
        off += (size_t)s.n1 * 4;
        s.total = (off + 15) / 16 * 16;
        return s;
    }
};

__device__ __forceinline__ double block_sum(double v, double *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += scratch[w];
    return s;
}

template <typename TIn, bool GRAD, bool PRED>
__global__ void __launch_bounds__(kBlkThreads) local_block_kernel(
    const __grid_constant__ LocalArgs a, const TIn *__restrict__ x_ref, const TIn *__restrict__ y_ref,
    const TIn *__restrict__ x_pt, const TIn *__restrict__ y_pt, const int32_t *__restrict__ nbr,
    double *__restrict__ block_out, TIn *__restrict__ mean, TIn *__restrict__ var, int32_t *__restrict__ flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Hyp h = hyp_of(a);
    const BlockSmem L = BlockSmem::make(a.m, a.d);
    double *A = reinterpret_cast<double *>(smem_raw + L.a_off);
    double *xs = reinterpret_cast<double *>(smem_raw + L.xs_off);
    double *yv = reinterpret_cast<double *>(smem_raw + L.vec_off);
    double *z = yv + L.n1, *zw = z + L.n1, *bb = zw + L.n1, *vv = bb + L.n1, *tmp = vv + L.n1;
    double *scratch = tmp + L.n1;
    int32_t *ids = reinterpret_cast<int32_t *>(smem_raw + L.idx_off);
    const int m = a.m, n1 = L.n1, lda = L.lda, d = a.d, tid = threadIdx.x;
    const int nth = 1 + a.n_theta;
    double ll_acc = 0.0;
    double g_loc[4] = {0, 0, 0, 0};  // amp, const, noise, iso (thread partials)

    // per-feature length-scale terms are added to this CTA's output slots system by system
    double *o = block_out + (int64_t)blockIdx.x * nth;
    if (!PRED && tid < nth) o[tid] = 0.0;

    for (int64_t p = blockIdx.x; p < a.n_points; p += gridDim.x) {
        __syncthreads();
        for (int i = tid; i < n1; i += blockDim.x) {
            int32_t jj = -2;  // -2: the point itself (row m)
            if (i < m) {
                jj = nbr[p * m + i];
                if (jj < -1 || (int64_t)jj >= a.n_rows) {
                    flag_or(flags, NNGP_FLAG_BAD_INDEX);
                    jj = -1;
                }
            }
            ids[i] = jj;
        }
        __syncthreads();
        for (int e = tid; e < n1 * d; e += blockDim.x) {
            const int i = e / d, f = e - i * d;
            const int32_t jj = ids[i];
            const double s = h.inv_ls[a.ard ? f : 0];
            double v = 0.0;
            if (jj >= 0) v = (double)x_ref[(int64_t)jj * d + f] * s;
            else if (jj == -2) v = (double)x_pt[p * d + f] * s;
            xs[i * d + f] = v;
        }
        __syncthreads();
        // fill the lower triangle (i >= j) of the augmented matrix, point = row m
        for (int e = tid; e < n1 * n1; e += blockDim.x) {
            const int i = e / n1, jx = e - i * n1;
            if (jx > i) continue;
            const bool vi = ids[i] != -1, vj = ids[jx] != -1;
            double kv;
            if (vi && vj) {
                double r = 0.0;
                for (int f = 0; f < d; ++f) {
                    const double t = xs[i * d + f] - xs[jx * d + f];
                    r = fma(t, t, r);
                }
                kv = h.rbf * kern_s<true>(a.family, r) + h.cst;
                if (i == jx)
                    kv += h.noise + (((i == m && PRED) || (i < m && (int64_t)ids[i] >= a.alpha_below)) ? 0.0 : a.alpha);
            } else {
                kv = (i == jx) ? 1.0 : 0.0;
            }
            A[i * lda + jx] = kv;
        }
        __syncthreads();
        // right-looking Cholesky
        bool notpd = false;
        for (int k = 0; k < n1; ++k) {
            __syncthreads();  // the previous trailing update is complete
            const double piv = A[k * lda + k];
            if (!(piv > 0.0)) notpd = true;
            const double sq = sqrt(piv);
            const double inv = 1.0 / sq;
            __syncthreads();  // every thread has read the pivot before it is overwritten
            for (int i = k + 1 + tid; i < n1; i += blockDim.x) A[i * lda + k] *= inv;
            if (tid == 0) A[k * lda + k] = sq;
            __syncthreads();
            const int rem = n1 - k - 1;
            for (int e = tid; e < rem * rem; e += blockDim.x) {
                const int i = k + 1 + e / rem, jx = k + 1 + e % rem;
                if (jx <= i) A[i * lda + jx] = fma(-A[i * lda + k], A[jx * lda + k], A[i * lda + jx]);
            }
        }
        __syncthreads();
        if (notpd && tid == 0) flag_or(flags, NNGP_FLAG_NOT_PD);
        const double sigma = A[m * lda + m];
        const double s2 = sigma * sigma;
        if (PRED && a.weights_out) {
            // conditioning weights w = L^-T l (l: row m of the augmented factor), by warp 0
            if (tid < 32) {
                for (int k = m - 1; k >= 0; --k) {
                    double part = 0.0;
                    for (int jx = k + 1 + tid; jx < m; jx += 32) part = fma(A[jx * lda + k], zw[jx], part);
                    part = warp_sum(part);
                    if (tid == 0) zw[k] = (A[m * lda + k] - part) / A[k * lda + k];
                    __syncwarp();
                }
            }
            __syncthreads();
            for (int i = tid; i < m; i += blockDim.x) mean[p * m + i] = (TIn)zw[i];
            if (tid == 0) var[p] = (TIn)s2;
            __syncthreads();
            continue;
        }
        double wsum = 0.0, ll = 0.0;
        for (int i = tid; i < n1; i += blockDim.x) zw[i] = 0.0;
        for (int c = 0; c < a.ydim; ++c) {
            __syncthreads();
            for (int i = tid; i < m; i += blockDim.x) yv[i] = ids[i] >= 0 ? (double)y_ref[(int64_t)ids[i] * a.ydim + c] : 0.0;
            __syncthreads();
            // forward solve with warp 0: z = L_nn^-1 yv
            if (tid < 32) {
                for (int k = 0; k < m; ++k) {
                    double part = 0.0;
                    for (int jx = tid; jx < k; jx += 32) part = fma(A[k * lda + jx], z[jx], part);
                    part = warp_sum(part);
                    if (tid == 0) z[k] = (yv[k] - part) / A[k * lda + k];
                    __syncwarp();
                }
                double part = 0.0;
                for (int jx = tid; jx < m; jx += 32) part = fma(A[m * lda + jx], z[jx], part);
                part = warp_sum(part);
                if (tid == 0) tmp[0] = part;  // mu
            }
            __syncthreads();
            const double mu = tmp[0];
            if (PRED) {
                if (tid == 0) mean[p * a.ydim + c] = (TIn)mu;
            } else {
                const double res = (double)y_pt[p * a.ydim + c] - mu;
                ll += -0.5 * res * res / s2 - log(sigma) - kHalfLog2Pi;
                if (GRAD) {
                    const double rs = res / s2;
                    for (int i = tid; i < m; i += blockDim.x) zw[i] = fma(rs, z[i], zw[i]);
                    wsum += (res * rs - 1.0) / (2.0 * s2);
                }
            }
        }
        if (PRED) {
            if (tid == 0) var[p] = (TIn)s2;
            continue;
        }
        if (tid == 0) ll_acc += ll;
        if (!GRAD) continue;
        __syncthreads();
        // backward solves with warp 0: b = L^-T l, v = L^-T zw (l = row m of the factor)
        if (tid < 32) {
            for (int k = m - 1; k >= 0; --k) {
                double pb = 0.0, pv = 0.0;
                for (int jx = k + 1 + tid; jx < m; jx += 32) {
                    pb = fma(A[jx * lda + k], bb[jx], pb);
                    pv = fma(A[jx * lda + k], vv[jx], pv);
                }
                pb = warp_sum(pb);
                pv = warp_sum(pv);
                if (tid == 0) {
                    bb[k] = (A[m * lda + k] - pb) / A[k * lda + k];
                    vv[k] = (zw[k] - pv) / A[k * lda + k];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // G-weighted recomputed fill over pairs i >= j of the augmented matrix
        double t_amp = 0.0, t_cst = 0.0, t_noise = 0.0, t_iso = 0.0;
        for (int e = tid; e < n1 * n1; e += blockDim.x) {
            const int i = e / n1, jx = e - i * n1;
            if (jx > i) continue;
            if (ids[i] == -1 || ids[jx] == -1) continue;
            double G;
            if (i == m && jx == m) G = wsum;
            else if (i == m) G = 0.5 * vv[jx] - wsum * bb[jx];
            else G = wsum * bb[i] * bb[jx] - 0.5 * (bb[i] * vv[jx] + vv[i] * bb[jx]);
            const double wgt = (i == jx) ? 1.0 : 2.0;
            double r = 0.0;
            for (int f = 0; f < d; ++f) {
                const double t = xs[i * d + f] - xs[jx * d + f];
                r = fma(t, t, r);
            }
            const double s0 = kern_s<true>(a.family, r);
            t_amp += wgt * G * h.rbf * s0;
            t_cst += wgt * G;
            if (i == jx) t_noise += G;
            t_iso += wgt * G * h.rbf * kern_g<true>(a.family, r, s0) * r;
        }
        g_loc[0] += t_amp;
        g_loc[1] += t_cst;
        g_loc[2] += t_noise;
        g_loc[3] += t_iso;
        if (a.idx_ls >= 0 && a.ard) {
            for (int f = 0; f < d; ++f) {
                double acc = 0.0;
                for (int e = tid; e < n1 * n1; e += blockDim.x) {
                    const int i = e / n1, jx = e - i * n1;
                    if (jx >= i) continue;  // diagonal terms vanish (dx = 0)
                    if (ids[i] == -1 || ids[jx] == -1) continue;
                    double G;
                    if (i == m) G = 0.5 * vv[jx] - wsum * bb[jx];
                    else G = wsum * bb[i] * bb[jx] - 0.5 * (bb[i] * vv[jx] + vv[i] * bb[jx]);
                    double r = 0.0;
                    for (int ff = 0; ff < d; ++ff) {
                        const double t = xs[i * d + ff] - xs[jx * d + ff];
                        r = fma(t, t, r);
                    }
                    const double t = xs[i * d + f] - xs[jx * d + f];
                    acc += 2.0 * G * h.rbf * kern_g<true>(a.family, r, kern_s<true>(a.family, r)) * t * t;
                }
                const double s = block_sum(acc, scratch);
                if (tid == 0) o[1 + a.idx_ls + f] += s;
            }
        }
    }
    if (PRED) return;
    __syncthreads();
    const double s_ll = block_sum(ll_acc, scratch);
    if (tid == 0) o[0] = s_ll;
    if (GRAD) {
        const double s0 = block_sum(g_loc[0], scratch);
        const double s1 = block_sum(g_loc[1], scratch);
        const double s2v = block_sum(g_loc[2], scratch);
        const double s3 = block_sum(g_loc[3], scratch);
        if (tid == 0) {
            if (a.idx_rbf >= 0) o[1 + a.idx_rbf] += s0;
            if (a.idx_const >= 0) o[1 + a.idx_const] += h.cst * s1;
            if (a.idx_noise >= 0) o[1 + a.idx_noise] += h.noise * s2v;
            if (a.idx_ls >= 0 && !a.ard) o[1 + a.idx_ls] += s3;
        }
    }
}

// Fixed-order sum of the per-CTA partials: out[t] = sum_b block_out[b * nt + t].
__global__ void finalize_kernel(const double *__restrict__ block_out, int nblocks, int nt, double *__restrict__ out) {
    __shared__ double scratch[32];
    for (int t = 0; t < nt; ++t) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += block_out[(int64_t)b * nt + t];
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) out[t] = s;
    }
}

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
namespace {

int num_sms() {
    static int cached = 0;
    if (!cached) {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
            cached = v;
        else
            cached = kNumSMsB200;
    }
    return cached;
}

size_t block_smem_limit() { return 227 * 1024; }

constexpr size_t kCountBytes = 256;  // head of the log-likelihood workspace: the FP64 re-solve count

struct LocalPlan {
    bool warp = true;
    int grid = 0;
    int redo_grid = 0;  // CTAs of local_redo_kernel (their partials follow the main kernel's)
    size_t smem = 0;
    int nt = 1;
    size_t bits_off = 0;  // byte offset of the FP64 re-solve bitmask from the workspace head
    size_t ws_bytes = 0;
};

// f32: the launch runs the FP32-input kernels (their warp layout keeps the squared distances);
// sys4: and only FP32 systems (the fit step: 4-byte warp layout)
LocalPlan plan_local(int64_t n_points, int d, int m, int n_theta, bool grad, bool f32 = false, bool sys4 = false) {
    LocalPlan p;
    p.warp = m <= kWarpM;
    p.nt = 1 + (grad ? n_theta : 0);
    const int sms = num_sms();
    if (p.warp) {
        p.smem = WarpSmem::make(d, n_theta, f32, sys4).total * kLocWarps;
        const int64_t need = (n_points + kLocWarps - 1) / kLocWarps;
        p.grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * 8));
    } else {
        p.smem = BlockSmem::make(m, d).total;
        p.grid = (int)std::max<int64_t>(1, std::min<int64_t>(n_points, (int64_t)sms * 2));
    }
    // [256 bytes: the count of FP64 re-solves | per-CTA partials of the main kernel, then of the
    // re-solve kernel | the re-solve bitmask, one bit per point], plus 256 of alignment slack
    // (laid out for FP32 inputs whatever the dtype: the workspace size does not depend on it)
    const int64_t words = (n_points + 31) / 32;
    p.redo_grid = (int)std::max<int64_t>(1, std::min<int64_t>((words + kLocWarps - 1) / kLocWarps, (int64_t)sms * 8));
    p.bits_off = kCountBytes + align_up((size_t)(p.grid + p.redo_grid) * p.nt * sizeof(double), 256);
    p.ws_bytes = p.bits_off + align_up((size_t)words * sizeof(uint32_t), 256) + 256;
    return p;
}

nngp_status fill_args(LocalArgs &a, const nngp_kernel *k, int d, int ydim, int m, int64_t n_rows, int64_t n_points,
                      double pivot_tol, bool grad) {
    if (!k) return fail(NNGP_ERR_INVALID_ARGUMENT, "kernel parameters are null");
    if (d <= 0 || d > kMaxDimLocal) return fail(NNGP_ERR_UNSUPPORTED, "d must be in [1, 256]");
    if (ydim <= 0) return fail(NNGP_ERR_INVALID_ARGUMENT, "ydim must be >= 1");
    if (m < 0) return fail(NNGP_ERR_INVALID_ARGUMENT, "m must be >= 0");
    if (k->n_ls != 0 && k->n_ls != 1 && k->n_ls != d) return fail(NNGP_ERR_INVALID_ARGUMENT, "n_ls must be 0, 1 or d");
    if (k->n_ls > 0 && !k->length_scale) return fail(NNGP_ERR_INVALID_ARGUMENT, "length_scale is null");
    if (grad && (k->n_theta < 0 || k->n_theta > kMaxTheta)) return fail(NNGP_ERR_UNSUPPORTED, "n_theta out of range");
    if (m > kWarpM) {
        const size_t need = BlockSmem::make(m, d).total;
        if (need > block_smem_limit())
            return fail(NNGP_ERR_UNSUPPORTED, "m = " + std::to_string(m) + " with d = " + std::to_string(d) +
                                                  " needs more shared memory than one CTA has");
    }
    a.rbf = k->rbf_level;
    a.cst = k->const_value;
    a.noise = k->noise_level;
    a.alpha = k->alpha;
    a.pivot_abs = pivot_tol * std::fabs(k->rbf_level + k->const_value + k->noise_level + k->alpha);
    a.n_rows = n_rows;
    a.n_points = n_points;
    a.d = d;
    a.ydim = ydim;
    a.m = m;
    a.ard = k->n_ls == d && d > 1;
    a.alpha_below = n_rows;
    a.weights_out = 0;
    a.fp64_count = nullptr;
    a.redo_bits = nullptr;
    a.dev_params = k->dev_params;
    if (k->family < NNGP_FAMILY_RBF || k->family > NNGP_FAMILY_MATERN52)
        return fail(NNGP_ERR_INVALID_ARGUMENT, "kernel family must be one of NNGP_FAMILY_*");
    a.family = k->family;
    a.idx_rbf = grad ? k->idx_rbf_level : -1;
    a.idx_const = grad ? k->idx_const : -1;
    a.idx_noise = grad ? k->idx_noise : -1;
    a.idx_ls = grad ? k->idx_ls : -1;
    a.n_theta = grad ? k->n_theta : 0;
    auto chk = [&](int idx, int span) { return idx < 0 || idx + span <= a.n_theta; };
    if (grad && !(chk(a.idx_rbf, 1) && chk(a.idx_const, 1) && chk(a.idx_noise, 1) && chk(a.idx_ls, a.ard ? d : 1)))
        return fail(NNGP_ERR_INVALID_ARGUMENT, "a theta index is outside [0, n_theta)");
    for (int f = 0; f < kMaxDimLocal; ++f) a.inv_ls[f] = 1.0;
    if (k->n_ls > 0) {
        for (int f = 0; f < (a.ard ? d : 1); ++f) {
            const double l = k->length_scale[a.ard ? f : 0];
            if (!(l > 0.0)) return fail(NNGP_ERR_INVALID_ARGUMENT, "length scales must be > 0");
            a.inv_ls[f] = 1.0 / l;
        }
    }
    return NNGP_OK;
}

template <typename TIn, bool GRAD, bool PRED>
nngp_status launch_local(const LocalPlan &pl, const LocalArgs &a, const TIn *x_ref, const TIn *y_ref, const TIn *x_pt,
                         const TIn *y_pt, const int32_t *nbr, double *block_out, TIn *mean, TIn *var, int32_t *flags,
                         cudaStream_t stream) {
    if (pl.warp) {
        auto fn = a.family == NNGP_FAMILY_RBF ? local_warp_kernel<TIn, GRAD, PRED, false>
                                              : local_warp_kernel<TIn, GRAD, PRED, true>;
        NNGP_CUDA_TRY(ensure_smem_limit(reinterpret_cast<const void *>(fn), (int)pl.smem));
        fn<<<pl.grid, kLocWarps * 32, pl.smem, stream>>>(a, x_ref, y_ref, x_pt, y_pt, nbr, block_out, mean, var, flags);
    } else {
        auto fn = local_block_kernel<TIn, GRAD, PRED>;
        NNGP_CUDA_TRY(ensure_smem_limit(reinterpret_cast<const void *>(fn), (int)pl.smem));
        fn<<<pl.grid, kBlkThreads, pl.smem, stream>>>(a, x_ref, y_ref, x_pt, y_pt, nbr, block_out, mean, var, flags);
    }
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

template <typename TIn>
nngp_status loglik_impl(const TIn *x, const TIn *y, int64_t n, int d, int ydim, int64_t row_begin, int64_t rows,
                        const int32_t *nbr, int m, const nngp_kernel *k, int eval_gradient, double pivot_tol,
                        double *out, int32_t *flags, void *ws, size_t ws_bytes, cudaStream_t stream) {
    if (n < 0 || rows < 0 || row_begin < 0 || row_begin + rows > n)
        return fail(NNGP_ERR_INVALID_ARGUMENT, "loglik: rows outside [0, n)");
    if (!out) return fail(NNGP_ERR_INVALID_ARGUMENT, "loglik: out is null");
    const bool grad = eval_gradient != 0;
    LocalArgs a;
    nngp_status st = fill_args(a, k, d, ydim, m, n, rows, pivot_tol, grad);
    if (st != NNGP_OK) return st;
    const int nt = 1 + (grad ? a.n_theta : 0);
    if (rows == 0) {
        NNGP_CUDA_TRY(cudaMemsetAsync(out, 0, nt * sizeof(double), stream));
        if (ws && ws_bytes >= kCountBytes + 256)
            NNGP_CUDA_TRY(cudaMemsetAsync(reinterpret_cast<void *>(align_up(reinterpret_cast<uintptr_t>(ws), 256)), 0,
                                          sizeof(unsigned long long), stream));
        return NNGP_OK;
    }
    if (!x || !y || (m > 0 && !nbr)) return fail(NNGP_ERR_INVALID_ARGUMENT, "loglik: null input pointer");
    const LocalPlan pl = plan_local(rows, d, m, a.n_theta, grad, std::is_same<TIn, float>::value,
                                    std::is_same<TIn, float>::value);
    if (!ws || ws_bytes < pl.ws_bytes) return fail(NNGP_ERR_WORKSPACE, "loglik: workspace missing or too small");
    unsigned char *head = reinterpret_cast<unsigned char *>(align_up(reinterpret_cast<uintptr_t>(ws), 256));
    a.fp64_count = reinterpret_cast<unsigned long long *>(head);
    NNGP_CUDA_TRY(cudaMemsetAsync(a.fp64_count, 0, sizeof(unsigned long long), stream));
    double *block_out = reinterpret_cast<double *>(head + kCountBytes);
    const TIn *x_pt = x + row_begin * d;
    const TIn *y_pt = y + row_begin * ydim;
    // FP32 warp systems: the points that need the FP64 re-solve are marked, then re-solved by a
    // second kernel (its partials follow the main kernel's; finalize sums both in a fixed order)
    const bool redo = std::is_same<TIn, float>::value && pl.warp;
    if (redo) {
        a.redo_bits = reinterpret_cast<uint32_t *>(head + pl.bits_off);
        NNGP_CUDA_TRY(cudaMemsetAsync(a.redo_bits, 0, (size_t)((rows + 31) / 32) * sizeof(uint32_t), stream));
    }
    if (grad)
        st = launch_local<TIn, true, false>(pl, a, x, y, x_pt, y_pt, nbr, block_out, nullptr, nullptr, flags, stream);
    else
        st = launch_local<TIn, false, false>(pl, a, x, y, x_pt, y_pt, nbr, block_out, nullptr, nullptr, flags, stream);
    if (st != NNGP_OK) return st;
    int parts = pl.grid;
    if constexpr (std::is_same<TIn, float>::value) {
        if (redo) {
            double *redo_out = block_out + (size_t)pl.grid * pl.nt;
            auto fn = a.family == NNGP_FAMILY_RBF ? (grad ? local_redo_kernel<true, false> : local_redo_kernel<false, false>)
                                                  : (grad ? local_redo_kernel<true, true> : local_redo_kernel<false, true>);
            const int redo_smem = (int)(WarpSmem::make(d, a.n_theta, true).total * kLocWarps);  // FP64 systems
            NNGP_CUDA_TRY(ensure_smem_limit(reinterpret_cast<const void *>(fn), redo_smem));
            fn<<<pl.redo_grid, kLocWarps * 32, redo_smem, stream>>>(a, x, y, x_pt, y_pt, nbr, redo_out, flags);
            NNGP_CUDA_TRY(cudaGetLastError());
            parts += pl.redo_grid;
        }
    }
    finalize_kernel<<<1, 256, 0, stream>>>(block_out, parts, pl.nt, out);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

template <typename TIn>
nngp_status predict_impl(const TIn *xt, const TIn *yt, int64_t nt, const TIn *xq, int64_t nq, int d, int ydim,
                         const int32_t *nbr, int m, const nngp_kernel *k, double pivot_tol, TIn *mean, TIn *var,
                         int32_t *flags, cudaStream_t stream) {
    if (nt < 0 || nq < 0) return fail(NNGP_ERR_INVALID_ARGUMENT, "predict: negative size");
    LocalArgs a;
    nngp_status st = fill_args(a, k, d, ydim, m, nt, nq, pivot_tol, false);
    if (st != NNGP_OK) return st;
    if (nq == 0) return NNGP_OK;
    if (!xq || !mean || !var || (m > 0 && (!nbr || !xt || !yt))) return fail(NNGP_ERR_INVALID_ARGUMENT, "predict: null pointer");
    const LocalPlan pl = plan_local(nq, d, m, 0, false, std::is_same<TIn, float>::value);
    return launch_local<TIn, false, true>(pl, a, xt, yt, xq, nullptr, nbr, nullptr, mean, var, flags, stream);
}

// ---------------------------------------------------------------------------------------
// Predict conditioned on the training set and the earlier queries ('full', the sequential
// algorithm of base_nngpr.py:896-1030)
// ---------------------------------------------------------------------------------------
// Covariance between two earlier queries a != b as the reference tracks it: only the pairs
// where the later one has the earlier one among its neighbours hold a value (the sparse
// partial covariance, :923-930, :1002-1008); every other pair counts as 0.
__device__ __forceinline__ double full_pair_cov(const int32_t *__restrict__ nbr, const double *pc, int m, int64_t nt,
                                               int64_t a, int64_t b) {
    const int64_t hi = a > b ? a : b, lo = a > b ? b : a;
    for (int u = 0; u < m; ++u)
        if ((int64_t)nbr[hi * m + u] == nt + lo) return pc[hi * m + u];
    return 0.0;
}

// One warp walks the queries in order (query i may condition on queries < i).  Lane l owns
// neighbour slots l and l + 32: mean_i = sum_s w_is v_s (v = y of a training neighbour or the
// mean already predicted for a query neighbour); var_i = max(0, max(0, s2_i) + w_q^T C w_q) with
// C the covariance of the query neighbours (variances on the diagonal, tracked pairs elsewhere);
// the covariances of query i with its query neighbours, (C w)_s, are kept for later queries.
__global__ void __launch_bounds__(32) full_recursion_kernel(const int32_t *__restrict__ nbr,
                                                            const double *__restrict__ w,
                                                            const double *__restrict__ s2,
                                                            const double *__restrict__ y, int64_t nt, int64_t nq,
                                                            int m, int ydim, int want_var, double *mean, double *var,
                                                            double *pc, int32_t *__restrict__ flags) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x;
    for (int64_t i = 0; i < nq; ++i) {
        int32_t j[2];
        double ws[2];
        bool q[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int sl = lane + 32 * h;
            int32_t jj = sl < m ? nbr[i * m + sl] : -1;
            if (jj >= 0 && (int64_t)jj >= nt + i) {  // not an earlier point: treated as missing
                flag_or(flags, NNGP_FLAG_BAD_INDEX);
                jj = -1;
            }
            j[h] = jj;
            ws[h] = (sl < m && jj >= 0) ? w[i * m + sl] : 0.0;
            q[h] = jj >= 0 && (int64_t)jj >= nt;  // a query neighbour
        }
        for (int c = 0; c < ydim; ++c) {
            double acc = 0.0;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (j[h] < 0) continue;
                const double v = q[h] ? mean[((int64_t)j[h] - nt) * ydim + c] : y[(int64_t)j[h] * ydim + c];
                acc = fma(ws[h], v, acc);
            }
            const double mu = warp_sum(acc);
            if (lane == 0) mean[i * ydim + c] = mu;
        }
        if (want_var) {
            double cw[2] = {0.0, 0.0};
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (q[h]) cw[h] = var[(int64_t)j[h] - nt] * ws[h];
            for (int t = 0; t < m; ++t) {
                const int32_t jt = __shfl_sync(FULL, t < 32 ? j[0] : j[1], t & 31);
                const double wt = __shfl_sync(FULL, t < 32 ? ws[0] : ws[1], t & 31);
                if (jt < 0 || (int64_t)jt < nt) continue;
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    if (q[h] && t != lane + 32 * h)
                        cw[h] += full_pair_cov(nbr, pc, m, nt, (int64_t)j[h] - nt, (int64_t)jt - nt) * wt;
            }
            const double quad = warp_sum(ws[0] * cw[0] + ws[1] * cw[1]);
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (lane + 32 * h < m) pc[i * m + lane + 32 * h] = q[h] ? cw[h] : 0.0;
            if (lane == 0) {
                const double raw = s2[i] > 0.0 ? s2[i] : 0.0;
                const double vi = raw + quad;
                var[i] = vi > 0.0 ? vi : 0.0;
            }
        }
        __syncwarp();  // this query's mean, variance and covariances are visible to the next ones
    }
}

// Samples conditioned on the training set and on the samples of the earlier queries (sample_y
// with conditioning_method='full', base_nngpr.py:691-750): sample_i = sum_s w_is v_s +
// max(0, sqrt(s2_i)) z_i, v the training y or the earlier query's sample of the same column.
// One warp walks the queries in order; lanes share the ydim * n_samples columns.
__global__ void __launch_bounds__(32) sample_recursion_kernel(const int32_t *__restrict__ nbr,
                                                              const double *__restrict__ w,
                                                              const double *__restrict__ s2,
                                                              const double *__restrict__ y, int64_t nt, int64_t nq,
                                                              int m, int ydim, int ns, const double *__restrict__ z,
                                                              double *out, int32_t *__restrict__ flags) {
    const int lane = threadIdx.x;
    const int cols = ydim * ns;
    for (int64_t i = 0; i < nq; ++i) {
        const double sig = s2[i] > 0.0 ? sqrt(s2[i]) : 0.0;
        for (int col = lane; col < cols; col += 32) {
            const int c = col / ns;
            double v = 0.0;
            for (int sl = 0; sl < m; ++sl) {
                const int32_t j = nbr[i * m + sl];
                if (j < 0) continue;
                if ((int64_t)j >= nt + i) {  // not an earlier point: treated as missing
                    flag_or(flags, NNGP_FLAG_BAD_INDEX);
                    continue;
                }
                const double val = (int64_t)j < nt ? y[(int64_t)j * ydim + c] : out[((int64_t)j - nt) * cols + col];
                v = fma(w[i * m + sl], val, v);
            }
            out[i * cols + col] = v + sig * z[i * cols + col];
        }
        __syncwarp();  // this query's samples are visible to the next ones
    }
}

// Predict with the dense predictive covariance (return_cov with 'full' conditioning,
// base_nngpr.py:989-1000): like full_recursion_kernel, but the covariance of every pair of
// queries is kept (cov, nq x nq, symmetric), so the query neighbours' covariance C is dense:
// cov[i, j] = sum_s w_is cov[a_s, j] over the query neighbours a_s of i, for every j < i, and
// cov[i, i] = max(0, max(0, s2_i) + w^T C w).  One CTA walks the queries in order; its threads
// share the row.
constexpr int kCovThreads = 256;
__global__ void __launch_bounds__(kCovThreads) cov_recursion_kernel(const int32_t *__restrict__ nbr,
                                                                    const double *__restrict__ w,
                                                                    const double *__restrict__ s2,
                                                                    const double *__restrict__ y, int64_t nt,
                                                                    int64_t nq, int m, int ydim, double *mean,
                                                                    double *cov, int32_t *__restrict__ flags) {
    __shared__ int64_t sa[64];   // query position of each slot's neighbour, or -1
    __shared__ int32_t sj[64];   // neighbour index (-1: missing)
    __shared__ double sw[64];
    __shared__ double svar;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t i = 0; i < nq; ++i) {
        if (tid < 64) {
            int32_t j = tid < m ? nbr[i * m + tid] : -1;
            if (j >= 0 && (int64_t)j >= nt + i) {
                flag_or(flags, NNGP_FLAG_BAD_INDEX);
                j = -1;
            }
            sj[tid] = j;
            sw[tid] = (tid < m && j >= 0) ? w[i * m + tid] : 0.0;
            sa[tid] = (j >= 0 && (int64_t)j >= nt) ? (int64_t)j - nt : -1;
        }
        __syncthreads();
        if (warp == 0) {
            for (int c = 0; c < ydim; ++c) {
                double acc = 0.0;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int sl = lane + 32 * h;
                    const int32_t j = sj[sl];
                    if (j < 0) continue;
                    const double v = sa[sl] >= 0 ? mean[sa[sl] * ydim + c] : y[(int64_t)j * ydim + c];
                    acc = fma(sw[sl], v, acc);
                }
                const double mu = warp_sum(acc);
                if (lane == 0) mean[i * ydim + c] = mu;
            }
            double part = 0.0;  // sum over this lane's slots s of w_s (C w)_s
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int sl = lane + 32 * h;
                const int64_t a = sa[sl];
                if (a < 0) continue;
                double cw = 0.0;
                for (int t = 0; t < m; ++t) {
                    const int64_t b = sa[t];
                    if (b >= 0) cw += cov[a * nq + b] * sw[t];
                }
                part = fma(sw[sl], cw, part);
            }
            const double quad = warp_sum(part);
            if (lane == 0) {
                const double raw = s2[i] > 0.0 ? s2[i] : 0.0;
                const double vi = raw + quad;
                svar = vi > 0.0 ? vi : 0.0;
            }
        }
        for (int64_t jj = tid; jj < i; jj += blockDim.x) {
            double r = 0.0;
            for (int t = 0; t < m; ++t) {
                const int64_t b = sa[t];
                if (b >= 0) r += sw[t] * cov[b * nq + jj];
            }
            cov[i * nq + jj] = r;
            cov[jj * nq + i] = r;
        }
        __syncthreads();
        if (tid == 0) cov[i * nq + i] = svar;
        __syncthreads();  // row i (and the diagonal) are complete before query i + 1 reads them
    }
}

size_t predict_full_workspace(int64_t nq, int m) { return (size_t)(2 * nq * (int64_t)m + nq) * sizeof(double) + 256; }

// samples == false: predict (mean, and var when want_var; with dense_cov, var receives the
// nq x nq covariance); samples == true: want_var holds n_samples, z the standard normals and
// mean receives the samples.
nngp_status predict_full_f64(const double *x_full, const double *y_train, int64_t nt, int64_t nq, int d, int ydim,
                             const int32_t *nbr, int m, const nngp_kernel *k, int want_var, double *mean, double *var,
                             int32_t *flags, void *ws, size_t ws_bytes, cudaStream_t stream, bool samples = false,
                             const double *z = nullptr, bool dense_cov = false) {
    if (nt < 0 || nq < 0) return fail(NNGP_ERR_INVALID_ARGUMENT, "predict_full: negative size");
    if (m < 1 || m > 2 * kWarpM) return fail(NNGP_ERR_UNSUPPORTED, "predict_full: num_nn must be in [1, 64]");
    LocalArgs a;
    nngp_status st = fill_args(a, k, d, ydim, m, nt + nq, nq, 0.0, false);
    if (st != NNGP_OK) return st;
    if (nq == 0) return NNGP_OK;
    if (samples && (want_var < 1 || !z)) return fail(NNGP_ERR_INVALID_ARGUMENT, "sample_full: n_samples >= 1 and z");
    if (!x_full || !mean || (want_var && !samples && !var) || !nbr || (nt > 0 && !y_train))
        return fail(NNGP_ERR_INVALID_ARGUMENT, "predict_full: null pointer");
    if (!ws || ws_bytes < predict_full_workspace(nq, m))
        return fail(NNGP_ERR_WORKSPACE, "predict_full: workspace missing or too small");
    double *wts = reinterpret_cast<double *>(align_up(reinterpret_cast<uintptr_t>(ws), 256));
    double *s2 = wts + nq * (int64_t)m;
    double *pc = s2 + nq;
    a.alpha_below = nt;  // alpha on training neighbours only (base_nngpr.py:952-954)
    a.weights_out = 1;
    const LocalPlan pl = plan_local(nq, d, m, 0, false);
    st = launch_local<double, false, true>(pl, a, x_full, y_train, x_full + nt * d, nullptr, nbr, nullptr, wts, s2,
                                           flags, stream);
    if (st != NNGP_OK) return st;
    if (samples) {
        sample_recursion_kernel<<<1, 32, 0, stream>>>(nbr, wts, s2, y_train, nt, nq, m, ydim, want_var, z, mean,
                                                      flags);
    } else if (dense_cov) {
        cov_recursion_kernel<<<1, kCovThreads, 0, stream>>>(nbr, wts, s2, y_train, nt, nq, m, ydim, mean, var, flags);
    } else {
        full_recursion_kernel<<<1, 32, 0, stream>>>(nbr, wts, s2, y_train, nt, nq, m, ydim, want_var, mean, var, pc,
                                                    flags);
    }
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

}  // namespace

size_t predict_full_workspace_size(int64_t nq, int m) { return predict_full_workspace(nq, m); }

nngp_status predict_full(const double *x_full, const double *y_train, int64_t nt, int64_t nq, int d, int ydim,
                         const int32_t *nbr, int m, const nngp_kernel *k, int want_var, double *mean, double *var,
                         int32_t *flags, void *ws, size_t ws_bytes, cudaStream_t stream) {
    return predict_full_f64(x_full, y_train, nt, nq, d, ydim, nbr, m, k, want_var, mean, var, flags, ws, ws_bytes,
                            stream);
}

nngp_status predict_cov_full(const double *x_full, const double *y_train, int64_t nt, int64_t nq, int d, int ydim,
                             const int32_t *nbr, int m, const nngp_kernel *k, double *mean, double *cov, int32_t *flags,
                             void *ws, size_t ws_bytes, cudaStream_t stream) {
    return predict_full_f64(x_full, y_train, nt, nq, d, ydim, nbr, m, k, 1, mean, cov, flags, ws, ws_bytes, stream,
                            false, nullptr, true);
}

nngp_status sample_full(const double *x_full, const double *y_train, int64_t nt, int64_t nq, int d, int ydim,
                        const int32_t *nbr, int m, const nngp_kernel *k, int n_samples, const double *z, double *out,
                        int32_t *flags, void *ws, size_t ws_bytes, cudaStream_t stream) {
    return predict_full_f64(x_full, y_train, nt, nq, d, ydim, nbr, m, k, n_samples, out, nullptr, flags, ws, ws_bytes,
                            stream, true, z);
}

// ---------------------------------------------------------------------------------------
// Allocation-free variant of the FP64 log-likelihood (nngp_loglik_f64_noalloc)
// ---------------------------------------------------------------------------------------
// For callers that cannot allocate device memory (and so cannot supply the workspace of
// nngp_loglik_f64), the per-CTA partial sums live in this file-scope device array instead.
// Every GPU that loads the library holds it (kStaticBlocks * kStaticSlots doubles = 333 KiB)
// until the process exits.  All calls share it: calls that overlap on the GPU (different
// streams, or different host threads on one device) race on it.  Each launch writes every slot
// it later reads, so nothing has to be cleared between calls.
constexpr int kStaticBlocks = 1184;  // the local kernels' largest grid on a 148-SM B200
constexpr int kStaticSlots = 36;     // 1 + n_theta: up to 35 hyperparameters
static __device__ __align__(256) double g_loglik_scratch[kStaticBlocks * kStaticSlots];

namespace {
std::mutex g_scratch_mu;
double *g_scratch_addr[64] = {};

// Device address of g_loglik_scratch on the current device (looked up once per device;
// in host code the symbol itself is only a host-side stand-in, never a device address).
nngp_status static_scratch(double **out) {
    int dev = -1;
    NNGP_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(NNGP_ERR_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        NNGP_CUDA_TRY(cudaGetSymbolAddress(&p, g_loglik_scratch));
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return NNGP_OK;
}
}  // namespace

nngp_status loglik_f64_noalloc(const double *x, const double *y, int64_t n, int d, int ydim, const int32_t *nbr, int m,
                               const nngp_kernel *k, int eval_gradient, double *out, int32_t *flags,
                               cudaStream_t stream) {
    if (n < 0) return fail(NNGP_ERR_INVALID_ARGUMENT, "loglik_noalloc: n < 0");
    if (!out) return fail(NNGP_ERR_INVALID_ARGUMENT, "loglik_noalloc: out is null");
    const bool grad = eval_gradient != 0;
    LocalArgs a;
    nngp_status st = fill_args(a, k, d, ydim, m, n, n, 0.0, grad);
    if (st != NNGP_OK) return st;
    const int nt = 1 + (grad ? a.n_theta : 0);
    if (nt > kStaticSlots)
        return fail(NNGP_ERR_UNSUPPORTED, "loglik_noalloc: " + std::to_string(nt - 1) +
                                              " hyperparameters; the static scratch holds at most " +
                                              std::to_string(kStaticSlots - 1));
    if (n == 0) {
        NNGP_CUDA_TRY(cudaMemsetAsync(out, 0, nt * sizeof(double), stream));
        return NNGP_OK;
    }
    if (!x || !y || (m > 0 && !nbr)) return fail(NNGP_ERR_INVALID_ARGUMENT, "loglik_noalloc: null input pointer");
    double *block_out = nullptr;
    st = static_scratch(&block_out);
    if (st != NNGP_OK) return st;
    LocalPlan pl = plan_local(n, d, m, a.n_theta, grad);
    pl.grid = std::min(pl.grid, kStaticBlocks);  // the kernels stride over the points
    if (grad)
        st = launch_local<double, true, false>(pl, a, x, y, x, y, nbr, block_out, nullptr, nullptr, flags, stream);
    else
        st = launch_local<double, false, false>(pl, a, x, y, x, y, nbr, block_out, nullptr, nullptr, flags, stream);
    if (st != NNGP_OK) return st;
    finalize_kernel<<<1, 256, 0, stream>>>(block_out, pl.grid, pl.nt, out);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

size_t loglik_workspace(int64_t n, int d, int ydim, int m, int n_theta) {
    (void)ydim;
    return plan_local(std::max<int64_t>(n, 1), std::max(d, 1), m, std::max(n_theta, 0), true).ws_bytes;
}

nngp_status loglik_f32(const float *x, const float *y, int64_t n, int d, int ydim, const int32_t *nbr, int m,
                       const nngp_kernel *k, int eval_gradient, double pivot_tol, double *out, int32_t *flags, void *ws,
                       size_t ws_bytes, cudaStream_t stream) {
    return loglik_impl<float>(x, y, n, d, ydim, 0, n, nbr, m, k, eval_gradient, pivot_tol, out, flags, ws, ws_bytes,
                              stream);
}
nngp_status loglik_f64(const double *x, const double *y, int64_t n, int d, int ydim, const int32_t *nbr, int m,
                       const nngp_kernel *k, int eval_gradient, double pivot_tol, double *out, int32_t *flags, void *ws,
                       size_t ws_bytes, cudaStream_t stream) {
    return loglik_impl<double>(x, y, n, d, ydim, 0, n, nbr, m, k, eval_gradient, pivot_tol, out, flags, ws, ws_bytes,
                               stream);
}
nngp_status loglik_rows_f32(const float *x, const float *y, int64_t n, int d, int ydim, int64_t r0, int64_t rc,
                            const int32_t *nbr, int m, const nngp_kernel *k, int eval_gradient, double pivot_tol,
                            double *out, int32_t *flags, void *ws, size_t ws_bytes, cudaStream_t stream) {
    return loglik_impl<float>(x, y, n, d, ydim, r0, rc, nbr, m, k, eval_gradient, pivot_tol, out, flags, ws, ws_bytes,
                              stream);
}
nngp_status loglik_rows_f64(const double *x, const double *y, int64_t n, int d, int ydim, int64_t r0, int64_t rc,
                            const int32_t *nbr, int m, const nngp_kernel *k, int eval_gradient, double pivot_tol,
                            double *out, int32_t *flags, void *ws, size_t ws_bytes, cudaStream_t stream) {
    return loglik_impl<double>(x, y, n, d, ydim, r0, rc, nbr, m, k, eval_gradient, pivot_tol, out, flags, ws, ws_bytes,
                               stream);
}
nngp_status predict_f32(const float *xt, const float *yt, int64_t nt, const float *xq, int64_t nq, int d, int ydim,
                        const int32_t *nbr, int m, const nngp_kernel *k, double pivot_tol, float *mean, float *var,
                        int32_t *flags, cudaStream_t stream) {
    return predict_impl<float>(xt, yt, nt, xq, nq, d, ydim, nbr, m, k, pivot_tol, mean, var, flags, stream);
}
nngp_status predict_f64(const double *xt, const double *yt, int64_t nt, const double *xq, int64_t nq, int d, int ydim,
                        const int32_t *nbr, int m, const nngp_kernel *k, double pivot_tol, double *mean, double *var,
                        int32_t *flags, cudaStream_t stream) {
    return predict_impl<double>(xt, yt, nt, xq, nq, d, ydim, nbr, m, k, pivot_tol, mean, var, flags, stream);
}

// ---------------------------------------------------------------------------------------
// Hyperparameter values from a device theta (nngp_theta_params)
// ---------------------------------------------------------------------------------------
struct ThetaMap {
    int idx_rbf, idx_const, idx_noise, idx_ls, n_ls, d;
    double rbf, cst, noise, alpha, pivot_tol;  // the fixed values (used where the index is -1)
    double ls[kMaxDimLocal];                   // fixed length scales (idx_ls = -1)
};

// One CTA: out = [rbf, cst, noise, pivot_abs, 1/l_0 .. 1/l_{d-1}, l_0 .. l_{d-1}], the values
// fill_args computes on the host from kernel.clone_with_theta(theta).
__global__ void __launch_bounds__(256) theta_params_kernel(const __grid_constant__ ThetaMap t,
                                                           const double *__restrict__ theta,
                                                           double *__restrict__ out) {
    const double rbf = t.idx_rbf >= 0 ? exp(theta[t.idx_rbf]) : t.rbf;
    const double cst = t.idx_const >= 0 ? exp(theta[t.idx_const]) : t.cst;
    const double noise = t.idx_noise >= 0 ? exp(theta[t.idx_noise]) : t.noise;
    if (threadIdx.x == 0) {
        out[0] = rbf;
        out[1] = cst;
        out[2] = noise;
        out[3] = t.pivot_tol * fabs(rbf + cst + noise + t.alpha);
    }
    for (int f = threadIdx.x; f < t.d; f += blockDim.x) {
        const int q = t.n_ls > 1 ? f : 0;
        const double l = t.n_ls == 0 ? 1.0 : (t.idx_ls >= 0 ? exp(theta[t.idx_ls + q]) : t.ls[q]);
        out[4 + f] = 1.0 / l;
        out[4 + t.d + f] = l;
    }
}

nngp_status theta_params(const nngp_kernel *k, const double *theta_dev, int d, double pivot_tol, double *out,
                         cudaStream_t stream) {
    if (!k || !theta_dev || !out) return fail(NNGP_ERR_INVALID_ARGUMENT, "theta_params: null pointer");
    if (d <= 0 || d > kMaxDimLocal) return fail(NNGP_ERR_UNSUPPORTED, "theta_params: d must be in [1, 256]");
    if (k->n_ls != 0 && k->n_ls != 1 && k->n_ls != d)
        return fail(NNGP_ERR_INVALID_ARGUMENT, "theta_params: n_ls must be 0, 1 or d");
    ThetaMap t{};
    t.idx_rbf = k->idx_rbf_level;
    t.idx_const = k->idx_const;
    t.idx_noise = k->idx_noise;
    t.idx_ls = k->n_ls > 0 ? k->idx_ls : -1;
    t.n_ls = k->n_ls;
    t.d = d;
    t.rbf = k->rbf_level;
    t.cst = k->const_value;
    t.noise = k->noise_level;
    t.alpha = k->alpha;
    t.pivot_tol = pivot_tol;
    const int spans[4] = {1, 1, 1, t.n_ls > 1 ? t.n_ls : 1};
    const int idx[4] = {t.idx_rbf, t.idx_const, t.idx_noise, t.idx_ls};
    for (int i = 0; i < 4; ++i)
        if (idx[i] >= 0 && idx[i] + spans[i] > k->n_theta)
            return fail(NNGP_ERR_INVALID_ARGUMENT, "theta_params: a theta index is outside [0, n_theta)");
    if (k->n_ls > 0 && t.idx_ls < 0) {
        if (!k->length_scale) return fail(NNGP_ERR_INVALID_ARGUMENT, "theta_params: length_scale is null");
        for (int f = 0; f < k->n_ls; ++f) t.ls[f] = k->length_scale[f];
    }
    theta_params_kernel<<<1, 256, 0, stream>>>(t, theta_dev, out);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

}  // namespace nngp
