// Per-particle arithmetic of the packing step, shared by the CUDA kernels
// (rcpg_kernels.cu) and by the host-side emulation used in the CPU tests.
//
// Every product and sum goes through x*() helpers that never contract into
// FMA (device: __dmul_rn/__dadd_rn/...; host builds use -ffp-contract=off),
// so each value rounds exactly as in the reference engine's portable build
// (python_code/python/src/core/rcp_generator.cpp, "ENG" below).
//
// Position layout ("pos"): particle-major, stride P = pos_stride(ndim) doubles:
//   pos[i*P + d] = x_d (d < ndim), pos[i*P + ndim] = D0_i (growth-free diameter).
// The current diameter is always D0_i * kappa, a single rounding identical to
// the reference's D[i] = D0[i] * kappa (ENG:5733).
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define RCPG_HD __host__ __device__ __forceinline__
#define RCPG_UNROLL _Pragma("unroll")
#else
#define RCPG_HD inline
#define RCPG_UNROLL
#endif

namespace rcpg {

constexpr int kMaxDim = 8;

RCPG_HD constexpr int pos_stride(int ndim) { return (ndim + 2) & ~1; }

// ---- uncontracted IEEE double arithmetic --------------------------------
RCPG_HD double xmul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
RCPG_HD double xadd(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
RCPG_HD double xsub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
RCPG_HD double xdiv(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
RCPG_HD double xsqrt(double a) {
#if defined(__CUDA_ARCH__)
    return __dsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}
RCPG_HD double xrint(double a) {
#if defined(__CUDA_ARCH__)
    return rint(a);
#else
    return std::nearbyint(a);
#endif
}
RCPG_HD double xabs(double a) { return a < 0.0 ? -a : (a == 0.0 ? 0.0 : a); }

// Minimum image of one component: dd - nearbyint(dd*inv_box)*box (ENG:4097, :3282).
RCPG_HD double mic(double dd, double inv_box, double box) {
    return xsub(dd, xmul(xrint(xmul(dd, inv_box)), box));
}

// Geometry shared by every kernel of one packing.
struct Geometry {
    int ndim;
    int circle_k;        // -walls[0] when walls[0] < 0, else 0
    int any_flat_wall;   // some walls[d] == 1
    std::int8_t walls[kMaxDim];
    double box[kMaxDim];
    double inv_box[kMaxDim];  // 1.0 / box[d], as the reference precomputes it
};

// ---- pair shell test (neighbour-list membership) --------------------------
// Full-refresh membership of the pair of particles at xi, xj: MIC d2 < r_c^2,
//   r_c = (D_lo + D_hi)*0.5 + t                       for ndim <= 3 (kd-tree, ENG:3296)
//   r_c = D_lo*0.5 + t + (double)(float)(D_hi*0.5)     for ndim > 3  (sort+walk, ENG:1357)
// with D_lo / D_hi the diameters of the lower / higher particle index. d2 is
// symmetric bit for bit (the minimum image of -a is exactly -(image of a)),
// and so is r_c for ndim <= 3; only the ndim > 3 cutoff depends on the order.
template <int ND>
RCPG_HD double shell_cut(double D_lo, double D_hi, double t_shell) {
    if (ND <= 3) return xadd(xmul(xadd(D_lo, D_hi), 0.5), t_shell);
    const float half_f = static_cast<float>(xmul(D_hi, 0.5));
    return xadd(xadd(xmul(D_lo, 0.5), t_shell), static_cast<double>(half_f));
}

template <int ND>
RCPG_HD bool in_shell(const double* xi, const double* xj, double D_lo, double D_hi,
                      const double* box, const double* inv_box, double t_shell) {
    double d2 = 0.0;
    RCPG_UNROLL
    for (int d = 0; d < ND; ++d) {
        const double dd = mic(xsub(xj[d], xi[d]), inv_box[d], box[d]);
        d2 = xadd(d2, xmul(dd, dd));
    }
    double r_c;
    if (ND <= 3) {
        r_c = xadd(xmul(xadd(D_lo, D_hi), 0.5), t_shell);
    } else {
        const float half_f = static_cast<float>(xmul(D_hi, 0.5));
        r_c = xadd(xadd(xmul(D_lo, 0.5), t_shell), static_cast<double>(half_f));
    }
    return d2 < xmul(r_c, r_c);
}

// Scalar sums of one force evaluation (get_forces_nd_3, ENG:3597-4269).
// pair_*: over overlapping list pairs, each pair counted once (from its lower
// index). wall_*: flat hard walls and the curved container (ENG:4198-4257).
struct ForceSums {
    double pair_U, pair_Lc, pair_dk, pair_Fm, pair_maxov;
    double wall_U, wall_dk, wall_Fm;
    double sum_mag;     // sum of |F_i| over |F_i|^2 > 1e-16 (compute_mean_force, ENG:769-803)
    double sum_D;       // sum of current diameters (ENG:4262-4265)
    unsigned long long pair_count, wall_count, mag_count;
};

RCPG_HD void sums_zero(ForceSums& s) {
    s.pair_U = s.pair_Lc = s.pair_dk = s.pair_Fm = s.pair_maxov = 0.0;
    s.wall_U = s.wall_dk = s.wall_Fm = 0.0;
    s.sum_mag = s.sum_D = 0.0;
    s.pair_count = s.wall_count = s.mag_count = 0ull;
}

// Per-pair terms in the reference's accumulation order, for the exact
// (one-thread order) reduction: overlap, r_ij, r_ij*(dist - r_ij), F_mag.
struct PairTerms {
    double U, Lc, dk, Fm;
};

// MIC displacement dx = x_j - x_i and its squared length, accumulated in the
// reference's order (ENG:4097-4104); the shell test and the force share it.
template <int ND>
RCPG_HD double pair_disp(const double* xi, const double* xj, const double* box, const double* inv_box,
                         double* dx) {
    double d2 = 0.0;
RCPG_UNROLL
    for (int d = 0; d < ND; ++d) {
        dx[d] = mic(xsub(xj[d], xi[d]), inv_box[d], box[d]);
        d2 = xadd(d2, xmul(dx[d], dx[d]));
    }
    return d2;
}

// Force and scalar terms of an overlapping pair (d2 < r_ij^2) from its
// displacement, FP64 as in the reference (ENG:4105-4139).
template <int ND>
RCPG_HD void pair_terms_f64(const double* dx, double d2, double r_ij, double* fi, PairTerms& pt) {
    const double dist = xsqrt(d2);
    const double F_mag = -xsub(xdiv(r_ij, dist), 1.0);
RCPG_UNROLL
    for (int d = 0; d < ND; ++d) fi[d] = xadd(fi[d], xmul(F_mag, dx[d]));
    pt.U = xsub(1.0, xdiv(dist, r_ij));
    pt.Lc = r_ij;
    pt.dk = xmul(r_ij, xsub(dist, r_ij));
    pt.Fm = F_mag;
}

#if defined(__CUDACC__)
// ---- mixed-precision pair arithmetic (graph mode, pair_precision = mixed) --
// Differences are formed in FP64 and rounded to FP32; everything after that
// is FP32. Both directions of a pair see exactly negated displacements and the
// same d2, so both agree on membership and overlap and the forces cancel.

// Relative widening of the FP32 shell test (r_c^2): it covers the rounding of
// d2 and r_c in FP32 (about 1e-6 relative), so a row holds every pair of the
// FP64 shell; the few extra pairs just outside it are harmless (the forces
// count overlapping pairs only).
constexpr float kShellMarginF = 1.00001f;

// dx = x_j - x_i in FP64, rounded to FP32, with the minimum image taken by one
// box length when |dx| exceeds half the box (pairs never reach 1.5 boxes).
// Returns d2 in FP32.
template <int ND>
__device__ __forceinline__ float mixed_disp(const double* xi, const double* xj, const double* box,
                                            const float* half_box, float* dxf) {
    float d2 = 0.0f;
RCPG_UNROLL
    for (int d = 0; d < ND; ++d) {
        double dd = xsub(xj[d], xi[d]);
        float f = __double2float_rn(dd);
        if (fabsf(f) > half_box[d]) {
            dd = f > 0.0f ? xsub(dd, box[d]) : xadd(dd, box[d]);
            f = __double2float_rn(dd);
        }
        dxf[d] = f;
        d2 = __fmaf_rn(f, f, d2);
    }
    return d2;
}

// Force and scalar terms of an overlapping pair (d2 < rsum^2, rsum = r_ij) in
// FP32 (ENG:4105-4139 with FP32 operands); the force is added to the FP32
// per-particle sum fi, the scalar terms go to the FP64 accumulators. The
// overlap-dependent terms carry a relative error of about 1e-7 / overlap.
// The scalar terms of the FP32 pair path, kept in FP32: the per-particle sums
// of that path are FP32, so the terms never need an FP64 round trip.
struct PairTermsF {
    float U, Lc, dk, Fm;
};

template <int ND>
__device__ __forceinline__ void pair_terms_mixed_f(const float* dxf, float d2, float rsum, float* fi,
                                                   PairTermsF& pt) {
    const float inv_dist = rsqrtf(d2);
    const float dist = d2 * inv_dist;
    const float F_mag = __fmaf_rn(-rsum, inv_dist, 1.0f);  // -(r/dist - 1)
RCPG_UNROLL
    for (int d = 0; d < ND; ++d) fi[d] = __fmaf_rn(F_mag, dxf[d], fi[d]);
    pt.U = 1.0f - __fdividef(dist, rsum);
    pt.Lc = rsum;
    pt.dk = rsum * (dist - rsum);
    pt.Fm = F_mag;
}

template <int ND>
__device__ __forceinline__ void pair_terms_mixed(const float* dxf, float d2, float rsum, float* fi,
                                                 PairTerms& pt) {
    PairTermsF f;
    pair_terms_mixed_f<ND>(dxf, d2, rsum, fi, f);
    pt.U = static_cast<double>(f.U);
    pt.Lc = static_cast<double>(f.Lc);
    pt.dk = static_cast<double>(f.dk);
    pt.Fm = static_cast<double>(f.Fm);
}
#endif

// One overlapping pair seen from particle i with partner j (dx = x_j - x_i
// after MIC). Returns false when the pair does not overlap. ENG:4086-4139.
template <int ND>
RCPG_HD bool pair_force(const double* xi, double Di, const double* xj, double Dj,
                        const Geometry& g, double* fi, PairTerms& pt) {
    const double r_ij = xmul(0.5, xadd(Di, Dj));
    double dx[ND];
    const double d2 = pair_disp<ND>(xi, xj, g.box, g.inv_box, dx);
    if (!(d2 < xmul(r_ij, r_ij))) return false;
    pair_terms_f64<ND>(dx, d2, r_ij, fi, pt);
    return true;
}

// Flat walls and the curved container acting on particle i, added to its
// force after all pair terms, in the reference's order (ENG:4198-4257:
// axes ascending, wall 0 then wall 1, then the container). The scalar
// contributions are added in that same order to the three wall_* sums.
template <int ND, typename CountT>
RCPG_HD void wall_forces(const double* xi, double Di, const Geometry& g, double* fi,
                         double& U, double& dk, double& Fm, CountT& count) {
    if (g.any_flat_wall) {
RCPG_UNROLL
        for (int d = 0; d < ND; ++d) {
            if (g.walls[d] != 1) continue;
            const double r = xdiv(Di, 2.0);
            for (int wall = 0; wall < 2; ++wall) {
                const double dxw = xsub(xmul(g.box[d], static_cast<double>(wall)), xi[d]);
                const double dist = xabs(dxw);
                if (dist < r) {
                    const double F_mag = xmul(-2.0, xsub(xdiv(r, dist), 1.0));
                    U = xadd(U, xmul(2.0, xsub(1.0, xdiv(dist, r))));
                    ++count;
                    fi[d] = xadd(fi[d], xmul(F_mag, dxw));
                    dk = xadd(dk, xmul(xmul(2.0, r), xsub(dist, r)));
                    Fm = xadd(Fm, F_mag);
                }
            }
        }
    }
    if (g.circle_k > 0) {
        // loops run over all ND axes with a guard so that xi / dxc keep
        // compile-time indices (the container spans the first tk axes)
        const int tk = g.circle_k < ND ? g.circle_k : ND;
        const double r = xdiv(Di, 2.0);
        const double R = xdiv(g.box[0], 2.0);
        double dij = 0.0;
        RCPG_UNROLL
        for (int M = 0; M < ND; ++M)
            if (M < tk) dij = xadd(dij, xmul(xsub(xi[M], R), xsub(xi[M], R)));
        dij = xsqrt(dij);
        double delta = xsub(R, dij);
        if (delta < r) {
            double dxc[ND];
            delta = dij;
            dij = 0.0;
            RCPG_UNROLL
            for (int M = 0; M < ND; ++M) {
                dxc[M] = 0.0;
                if (M < tk) {
                    dxc[M] = xmul(xabs(xsub(xdiv(R, delta), 1.0)), xsub(xi[M], R));
                    dij = xadd(dij, xmul(dxc[M], dxc[M]));
                }
            }
            dij = xsqrt(dij);
            const double F_mag = xmul(-2.0, xabs(xsub(xdiv(r, dij), 1.0)));
            U = xadd(U, xsub(1.0, xdiv(dij, r)));
            ++count;
            RCPG_UNROLL
            for (int M = 0; M < ND; ++M)
                if (M < tk) fi[M] = xadd(fi[M], xmul(F_mag, dxc[M]));
            dk = xadd(dk, xmul(xmul(2.0, r), xsub(dij, r)));
            Fm = xadd(Fm, F_mag);
        }
    }
}

// |F_i|^2 in the reference's order (ENG:787-791).
template <int ND>
RCPG_HD double force_norm2(const double* fi) {
    double d2 = 0.0;
RCPG_UNROLL
    for (int d = 0; d < ND; ++d) d2 = xadd(d2, xmul(fi[d], fi[d]));
    return d2;
}

// Particle ADAM + position step + single-box wrap for one coordinate
// (fused pass ENG:6499-6519; adam_update ENG:4322-4329).
RCPG_HD double adam_coord(double F, double& m, double& v, double x, double alpha, double inv_b1,
                          double inv_b2, double L) {
    const double mk = xsub(xmul(0.9, m), xmul(xsub(1.0, 0.9), F));
    const double vk = xadd(xmul(0.999, v), xmul(xmul(xsub(1.0, 0.999), F), F));
    m = mk;
    v = vk;
    const double mhk = xmul(mk, inv_b1);
    const double vhk = xmul(vk, inv_b2);
    double xv = xsub(x, xdiv(xmul(alpha, mhk), xadd(xsqrt(vhk), 1e-8)));
    if (xv >= L) xv = xsub(xv, L);
    else if (xv < 0) xv = xadd(xv, L);
    return xv;
}

// Growth-aware displacement trigger for one particle (ENG:6129-6145):
// D_last is the running minimum of D since the anchor, theta the budget.
RCPG_HD bool refresh_trigger(double d2, double D, double D_last, double theta) {
    const double growth_half = xmul(xsub(D, D_last), 0.5);
    const double budget = xsub(theta, growth_half);
    return budget <= 0.0 || d2 > xmul(budget, budget);
}

// 21-bit-per-axis 3D Morton code of a position (ENG:1107-1160).
RCPG_HD std::uint64_t morton_spread21(std::uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x001F00000000FFFFull;
    v = (v | (v << 16)) & 0x001F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

RCPG_HD std::uint32_t morton_axis(double x, double box, double scale) {
    const double lim = xsub(box, 1e-12);
    double v = (x < lim) ? x : lim;  // std::min(box - 1e-12, x)
    v = (0.0 < v) ? v : 0.0;         // std::max(0.0, .)
    return static_cast<std::uint32_t>(xmul(v, scale));
}

// Order-preserving unsigned key of a double (x-column reorder key). Equal
// doubles (including -0.0 and +0.0) get equal keys, so ties fall back to the
// particle index as in the reference comparator (ENG:1083-1089).
RCPG_HD std::uint64_t double_order_key(double v) {
    if (v == 0.0) v = 0.0;
    std::uint64_t b;
#if defined(__CUDA_ARCH__)
    b = static_cast<std::uint64_t>(__double_as_longlong(v));
#else
    __builtin_memcpy(&b, &v, sizeof(b));
#endif
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

}  // namespace rcpg
