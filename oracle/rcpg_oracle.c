/* CPU restatement of the reference packing engine's per-step kernels.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the thing
 * measured or shipped. Built with -ffp-contract=off so every product and sum
 * rounds exactly as in the reference's portable build (no FMA contraction).
 * ENG = python_code/python/src/core/rcp_generator.cpp of the reference.
 * Declarations and layout conventions: rcpg_oracle.h.
 */
#include "rcpg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static int cmp_double(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/* ENG:2795-2846 (kd-tree D stats) and ENG:1204-1210 (sort+walk): the median
 * is the value at position N/2 of D in ascending order. */
double rcpo_t_shell(size_t N, const double* D) {
    double* s = (double*)malloc(N * sizeof(double));
    memcpy(s, D, N * sizeof(double));
    qsort(s, N, sizeof(double), cmp_double);
    const double dmin = s[0], dmax = s[N - 1], med = s[N / 2];
    free(s);
    double a = med * 1.02, b = dmin * 2.25;
    double m = a > b ? a : b;
    if (m > dmax) m = dmax;
    return m * 0.5;
}

/* Minimum-image component, ENG:3280-3290: dd -= nearbyint(dd*inv_box)*box. */
static inline double mic(double dd, double inv_box, double box) {
    return dd - nearbyint(dd * inv_box) * box;
}

size_t rcpo_pairs_full(size_t N, size_t ndim, const double* x, const double* D,
                       const double* box, double t_shell, uint32_t* counts, uint32_t* ids,
                       size_t cap) {
    double inv_box[16];
    for (size_t d = 0; d < ndim; ++d) inv_box[d] = 1.0 / box[d];
    size_t total = 0;
    for (size_t i = 0; i < N; ++i) {
        uint32_t c = 0;
        for (size_t j = i + 1; j < N; ++j) {
            double d2 = 0.0;
            for (size_t d = 0; d < ndim; ++d) {
                const double dd = mic(x[j * ndim + d] - x[i * ndim + d], inv_box[d], box[d]);
                d2 += dd * dd;
            }
            double r_c;
            if (ndim <= 3) {
                r_c = (D[i] + D[j]) * 0.5 + t_shell;               /* ENG:3296 */
            } else {
                const float half_f = (float)(D[j] * 0.5);          /* ENG:1286, :1357 */
                r_c = (D[i] * 0.5 + t_shell) + (double)half_f;
            }
            if (d2 >= r_c * r_c) continue;
            if (total < cap && ids) ids[total] = (uint32_t)j;
            ++total;
            ++c;
        }
        counts[i] = c;
    }
    return total;
}

void rcpo_forces(size_t N, size_t ndim, const double* x, const double* D, const double* box,
                 const int8_t* walls, const uint32_t* counts, const uint32_t* ids, double mu,
                 double* F, double* scalars) {
    const double K = 1.0;
    double inv_box[16];
    for (size_t d = 0; d < ndim; ++d) inv_box[d] = 1.0 / box[d];
    memset(F, 0, N * ndim * sizeof(double));
    double U = 0.0, Lc = 0.0, dkappa = 0.0, Fmean = 0.0, maxov = 0.0;
    size_t count_red = 0;
    /* pair loop, ENG:4086-4139 (scalar path; the AVX-512 variants are op-identical) */
    size_t k = 0;
    for (size_t i = 0; i < N; ++i) {
        const double Di = D[i];
        for (uint32_t q = 0; q < counts[i]; ++q) {
            const size_t j = ids[k++];
            const double r_ij = 0.5 * (Di + D[j]);
            double d2 = 0.0;
            double dxl[16];
            for (size_t d = 0; d < ndim; ++d) {
                const double delta = mic(x[j * ndim + d] - x[i * ndim + d], inv_box[d], box[d]);
                dxl[d] = delta;
                d2 += delta * delta;
            }
            const double r_ij_sq = r_ij * r_ij;
            if (d2 < r_ij_sq) {
                const double dist = sqrt(d2);
                const double F_mag = -K * (r_ij / dist - 1.0);
                const double overlap = 1.0 - dist / r_ij;
                U += overlap;
                ++count_red;
                Lc += r_ij;
                if (overlap > maxov) maxov = overlap;
                for (size_t d = 0; d < ndim; ++d) {
                    const double fcomp = F_mag * dxl[d];
                    F[i * ndim + d] += fcomp;
                    F[j * ndim + d] -= fcomp;
                }
                dkappa = dkappa + K * r_ij * (dist - r_ij);
                Fmean = Fmean + F_mag;
            }
        }
    }
    size_t count = 1 + count_red;                                   /* ENG:4195 */
    const int circle = walls[0] < 0;
    /* walls + curved container, ENG:4198-4257 (the `~no_walls` test is always true) */
    for (size_t i = 0; i < N; ++i) {
        for (size_t d = 0; d < ndim; ++d) {
            if (walls[d] == 1) {
                const double r_ij = D[i] / 2;
                for (size_t wall = 0; wall < 2; ++wall) {
                    const double dx = box[d] * (double)wall - x[i * ndim + d];
                    const double dist = fabs(dx);
                    if (dist < r_ij) {
                        const double F_mag = -2.0 * K * (r_ij / dist - 1.0);
                        U += 2.0 * (1.0 - dist / r_ij);
                        ++count;
                        const double fcomp = F_mag * dx;
                        F[i * ndim + d] += fcomp;
                        dkappa = dkappa + 2 * K * r_ij * (dist - r_ij);
                        Fmean = Fmean + F_mag;
                    }
                }
            }
        }
        if (circle) {
            const size_t t = (size_t)(-walls[0]);
            const double r_ij = D[i] / 2;
            const double R = box[0] / 2;
            double d_ij = 0;
            for (size_t M = 0; M < t; ++M)
                d_ij = d_ij + (x[i * ndim + M] - R) * (x[i * ndim + M] - R);
            d_ij = sqrt(d_ij);
            double delta = R - d_ij;
            if (delta < r_ij) {
                double dx[16];
                delta = d_ij;
                d_ij = 0;
                for (size_t M = 0; M < t; ++M) {
                    dx[M] = fabs(R / delta - 1) * (x[i * ndim + M] - R);
                    d_ij = d_ij + dx[M] * dx[M];
                }
                d_ij = sqrt(d_ij);
                const double F_mag = -2.0 * K * fabs(r_ij / d_ij - 1.0);
                U = U + (1 - d_ij / r_ij);
                ++count;
                for (size_t M = 0; M < t; ++M) F[i * ndim + M] = F[i * ndim + M] + F_mag * dx[M];
                dkappa = dkappa + 2 * K * r_ij * (d_ij - r_ij);
                Fmean = Fmean + F_mag;
            }
        }
    }
    /* finalise, ENG:4259-4268 */
    U = pow(U / (double)count, 2);
    Lc = Lc / (double)count;
    double sumD = 0.0;
    for (size_t i = 0; i < N; ++i) sumD += D[i];
    dkappa = dkappa + mu * sumD;
    Fmean = -Fmean / (double)count;
    scalars[0] = U;
    scalars[1] = maxov;
    scalars[2] = Lc;
    scalars[3] = Fmean;
    scalars[4] = dkappa;
    scalars[5] = (double)count;
}

double rcpo_mean_force(const double* F, size_t N, size_t ndim) {
    double sum_mag = 0.0;
    uint32_t count = 0;
    for (size_t i = 0; i < N; ++i) {
        double d2 = 0.0;
        for (size_t d = 0; d < ndim; ++d) d2 += F[i * ndim + d] * F[i * ndim + d];
        if (d2 > 1.0E-16) {
            sum_mag += sqrt(d2);
            ++count;
        }
    }
    const double mean_mag = sum_mag / (double)count;
    return mean_mag / sqrt((double)ndim);
}

void rcpo_adam_step(size_t N, size_t ndim, const double* F, double alpha, double inv_b1,
                    double inv_b2, const double* box, double* m, double* v, double* x) {
    const double beta1 = 0.9, beta2 = 0.999, eps = 1e-8;
    for (size_t k = 0; k < N; ++k) {
        for (size_t kk = 0; kk < ndim; ++kk) {
            const size_t idx = k * ndim + kk;
            const double Fk = F[idx];
            const double mk = beta1 * m[idx] - (1.0 - beta1) * Fk;
            const double vk = beta2 * v[idx] + (1.0 - beta2) * Fk * Fk;
            m[idx] = mk;
            v[idx] = vk;
            const double mhk = mk * inv_b1;
            const double vhk = vk * inv_b2;
            double xv = x[idx] - alpha * mhk / (sqrt(vhk) + eps);
            const double L = box[kk];
            if (xv >= L) xv -= L;
            else if (xv < 0) xv += L;
            x[idx] = xv;
        }
    }
}

double rcpo_kappa_step(double* st, double dkappa, double pow_b1, double pow_b2, double alpha,
                       double kappa) {
    const double beta1 = 0.9, beta2 = 0.999, eps = 1e-8;
    st[0] = beta1 * st[0] - (1 - beta1) * dkappa;
    st[1] = beta2 * st[1] + (1 - beta2) * (dkappa * dkappa);
    st[2] = st[0] / (1.0 - pow_b1);
    st[3] = st[1] / (1.0 - pow_b2);
    return kappa - alpha * st[2] / (sqrt(st[3]) + eps);
}

size_t rcpo_refresh_check(size_t N, size_t ndim, const double* x, double* x_last,
                          const double* D, double* D_last, double* theta_anchor,
                          double theta_new, uint8_t* refresh) {
    size_t n = 0;
    for (size_t k = 0; k < N; ++k) {
        const size_t base = k * ndim;
        double d2 = 0.0;
        for (size_t d = 0; d < ndim; ++d) {
            const double dd = x[base + d] - x_last[base + d];
            d2 += dd * dd;
        }
        if (D[k] < D_last[k]) D_last[k] = D[k];
        const double growth_half = (D[k] - D_last[k]) * 0.5;
        if (theta_anchor[k] > theta_new) theta_anchor[k] = theta_new;
        const double budget = theta_anchor[k] - growth_half;
        refresh[k] = 0;
        if (budget <= 0.0 || d2 > budget * budget) {
            refresh[k] = 1;
            for (size_t d = 0; d < ndim; ++d) x_last[base + d] = x[base + d];
            D_last[k] = D[k];
            theta_anchor[k] = theta_new;
            ++n;
        }
    }
    return n;
}

/* ---- reorder permutation ---- */
typedef struct {
    uint64_t key;
    uint32_t idx;
} keyidx;

static int cmp_keyidx(const void* a, const void* b) {
    const keyidx* p = (const keyidx*)a;
    const keyidx* q = (const keyidx*)b;
    if (p->key != q->key) return p->key < q->key ? -1 : 1;
    return (p->idx > q->idx) - (p->idx < q->idx);
}

typedef struct {
    double key;
    uint32_t idx;
} dblidx;

static int cmp_dblidx(const void* a, const void* b) {
    const dblidx* p = (const dblidx*)a;
    const dblidx* q = (const dblidx*)b;
    if (p->key < q->key) return -1;
    if (p->key > q->key) return 1;
    return (p->idx > q->idx) - (p->idx < q->idx);
}

/* Bit interleave of a 21-bit integer into every third bit (ENG:1111-1119). */
static uint64_t spread3(uint64_t v) {
    uint64_t r = 0;
    for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1ull) << (3 * b);
    return r;
}

void rcpo_reorder_perm(size_t N, size_t ndim, const double* x, const double* box, uint32_t* perm) {
    if (ndim == 3) {
        keyidx* c = (keyidx*)malloc(N * sizeof(keyidx));
        double sc[3];
        for (int d = 0; d < 3; ++d) sc[d] = ((double)(1u << 21) - 1.0) / box[d];
        for (size_t i = 0; i < N; ++i) {
            uint64_t code = 0;
            for (int d = 0; d < 3; ++d) {
                double lim = box[d] - 1e-12;
                double v = x[i * 3 + d];
                v = v < lim ? v : lim;      /* std::min(box - 1e-12, x) */
                v = 0.0 > v ? 0.0 : v;      /* std::max(0.0, .) */
                const uint32_t q = (uint32_t)(v * sc[d]);
                code |= spread3(q & 0x1FFFFFu) << d;
            }
            c[i].key = code;
            c[i].idx = (uint32_t)i;
        }
        qsort(c, N, sizeof(keyidx), cmp_keyidx);
        for (size_t k = 0; k < N; ++k) perm[k] = c[k].idx;
        free(c);
    } else {
        dblidx* c = (dblidx*)malloc(N * sizeof(dblidx));
        for (size_t i = 0; i < N; ++i) {
            c[i].key = x[i * ndim];
            c[i].idx = (uint32_t)i;
        }
        qsort(c, N, sizeof(dblidx), cmp_dblidx);
        for (size_t k = 0; k < N; ++k) perm[k] = c[k].idx;
        free(c);
    }
}

void rcpo_pair_caps(size_t N, size_t ndim, const double* D, uint32_t neighbor_max, uint32_t* caps) {
    static const uint32_t table[4] = {300, 750, 5500, 5500};
    if (neighbor_max == 0) {
        size_t idx = ndim >= 2 ? (ndim - 2 < 3 ? ndim - 2 : 3) : 0;
        neighbor_max = table[idx];
    }
    double dmin = D[0];
    for (size_t i = 1; i < N; ++i)
        if (D[i] < dmin) dmin = D[i];
    if (dmin <= 0.0) dmin = 1.0;
    const double scaling = (double)ndim / 3.0;
    const double omega = 1.0 + (double)ndim / 6.0;
    for (size_t i = 0; i < N; ++i) {
        const double cap_d = scaling * (50.0 * pow(D[i] / dmin, omega) + (double)neighbor_max);
        uint32_t cap = (uint32_t)ceil(cap_d);
        if ((uint64_t)cap > N) cap = (uint32_t)N;
        caps[i] = cap;
    }
}
