/*
 * v2m_unroll_oracle.c -- TEST INFRASTRUCTURE ONLY: the differentiable
 * relaxation unroll in FP64, serial, with its exact reverse-mode gradient, the
 * checker of the CUDA adjoint (trussnet_b200/csrc/v2m_adjoint.cu).
 *
 * The unroll (the reference has no adjoint; this is the relaxation step of
 * src/opencl/v2m_particle_body.cl:161-184 and the Jacobi branch of :898-900
 * with the discrete decisions frozen):
 *   h_i      = H(x_i): trilinear interpolation of the sizing grid G (m0 x m1 x m2
 *              values at x = (a cs0, b cs1, c cs2), x fastest), the point clamped
 *              to the grid's box
 *   F_i      = sum over i's list (frozen) of f (x_i - x_j), f = (l0 - l) / l for
 *              0 < l < l0, l0 = a_ij (h_i + h_j), a_ij = fsurf/2 if both nodes
 *              are non-INTERIOR else fscale/2
 *   c_i      = number of those active bars (piecewise constant)
 *   tape     = which bars are active at each step (one 24-bit mask per node and
 *              step): recorded by a forward pass, replayed by the backward pass
 *              and by forward passes that evaluate the same taped function (a
 *              replayed bar keeps f = (l0 - l) / l whatever its length), so the
 *              stiffness c_i, whose jumps make the untaped step discontinuous,
 *              is frozen
 *   x_i'     = x_i + dt F_i / max(c_i, 1)      (CORNER nodes stay)
 *              or, with taped constraints (dirs: per node a unit direction d
 *              and a kind), x_i' = x_i + P_i dt F_i / max(c_i, 1) with
 *              P_i = I - d d^T (kind 1, an INTERFACE node in its tangent plane)
 *              or d d^T (kind 2, a JUNCTION node along its line); the reverse
 *              step's increment adjoint is then P_i dt lam_i / max(c_i, 1)
 *   loss     = sum over every list entry (i, j) of (l_ij / hm_ij - 1)^2,
 *              hm_ij = (h_i + h_j) / 2, at the final positions.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define UK 24

typedef struct {
    int n;
    const int32_t* nbr;   /* row-major n x 24, local ids */
    const int32_t* nnb;
    const uint8_t* typ;
    int m[3];
    double cs[3];
    const double* G;
    double fscale, fsurf, dt;
    const double* dirs;   /* n x 4 (d, kind) or NULL */
} unroll_t;

/* v <- P_i v */
static void project(const unroll_t* U, int i, double* v) {
    if (!U->dirs) return;
    const double* d = U->dirs + 4 * (long)i;
    if (d[3] == 0.0) return;
    double t = v[0] * d[0] + v[1] * d[1] + v[2] * d[2];
    for (int k = 0; k < 3; ++k) v[k] = d[3] == 1.0 ? v[k] - t * d[k] : t * d[k];
}

/* h at x, its gradient (may be NULL), the 8 corner indices and weights */
static double size_at(const unroll_t* U, const double* x, double* grad, long* idx, double* w) {
    double u[3], f[3];
    int i0[3], inside[3];
    for (int d = 0; d < 3; ++d) {
        double v = x[d] / U->cs[d];
        inside[d] = v > 0.0 && v < (double)(U->m[d] - 1);
        if (v < 0.0) v = 0.0;
        if (v > (double)(U->m[d] - 1)) v = (double)(U->m[d] - 1);
        int a = (int)floor(v);
        if (a > U->m[d] - 2) a = U->m[d] > 1 ? U->m[d] - 2 : 0;
        i0[d] = a;
        u[d] = v;
        f[d] = v - a;
    }
    double c[8];
    for (int k = 0; k < 8; ++k) {
        int a = i0[0] + (k & 1), b = i0[1] + ((k >> 1) & 1), cc = i0[2] + (k >> 2);
        if (a >= U->m[0]) a = U->m[0] - 1;
        if (b >= U->m[1]) b = U->m[1] - 1;
        if (cc >= U->m[2]) cc = U->m[2] - 1;
        long id = a + (long)U->m[0] * (b + (long)U->m[1] * cc);
        c[k] = U->G[id];
        if (idx) idx[k] = id;
        double wx = (k & 1) ? f[0] : 1.0 - f[0], wy = ((k >> 1) & 1) ? f[1] : 1.0 - f[1], wz = (k >> 2) ? f[2] : 1.0 - f[2];
        if (w) w[k] = wx * wy * wz;
    }
    double h = 0.0;
    for (int k = 0; k < 8; ++k) {
        double wx = (k & 1) ? f[0] : 1.0 - f[0], wy = ((k >> 1) & 1) ? f[1] : 1.0 - f[1], wz = (k >> 2) ? f[2] : 1.0 - f[2];
        h += wx * wy * wz * c[k];
    }
    if (grad) {
        for (int d = 0; d < 3; ++d) {
            double g = 0.0;
            for (int k = 0; k < 8; ++k) {
                double wf[3] = { (k & 1) ? f[0] : 1.0 - f[0], ((k >> 1) & 1) ? f[1] : 1.0 - f[1], (k >> 2) ? f[2] : 1.0 - f[2] };
                double dsign = ((k >> d) & 1) ? 1.0 : -1.0;
                double prod = dsign;
                for (int e = 0; e < 3; ++e)
                    if (e != d) prod *= wf[e];
                g += prod * c[k];
            }
            grad[d] = inside[d] ? g / U->cs[d] : 0.0;
        }
    }
    (void)u;
    return h;
}

static double coef(const unroll_t* U, int i, int j) {
    return ((U->typ[i] != 0 && U->typ[j] != 0) ? U->fsurf : U->fscale) * 0.5;
}

static void step(const unroll_t* U, const double* x, double* y, double* h, uint32_t* mask, int replay) {
    for (int i = 0; i < U->n; ++i) h[i] = size_at(U, x + 3 * i, NULL, NULL, NULL);
    for (int i = 0; i < U->n; ++i) {
        if (U->typ[i] == 3) {
            memcpy(y + 3 * i, x + 3 * i, 3 * sizeof(double));
            continue;
        }
        double F[3] = { 0, 0, 0 };
        int c = 0;
        uint32_t bits = 0;
        for (int k = 0; k < U->nnb[i]; ++k) {
            int j = U->nbr[(long)i * UK + k];
            double e[3] = { x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2] };
            double l = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            double l0 = coef(U, i, j) * (h[i] + h[j]);
            int on = replay ? (int)((mask[i] >> k) & 1u) : (l < l0 && l > 0.0);
            if (!on) continue;
            bits |= 1u << k;
            double f = (l0 - l) / l;
            for (int d = 0; d < 3; ++d) F[d] += f * e[d];
            ++c;
        }
        if (!replay) mask[i] = bits;
        double s = U->dt / (c > 1 ? c : 1);
        double inc[3] = { s * F[0], s * F[1], s * F[2] };
        project(U, i, inc);
        for (int d = 0; d < 3; ++d) y[3 * i + d] = x[3 * i + d] + inc[d];
    }
}

static double loss_at(const unroll_t* U, const double* x, double* h) {
    for (int i = 0; i < U->n; ++i) h[i] = size_at(U, x + 3 * i, NULL, NULL, NULL);
    double L = 0.0;
    for (int i = 0; i < U->n; ++i)
        for (int k = 0; k < U->nnb[i]; ++k) {
            int j = U->nbr[(long)i * UK + k];
            double e[3] = { x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2] };
            double l = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            double r = l / (0.5 * (h[i] + h[j])) - 1.0;
            L += r * r;
        }
    return L;
}

/* lam += gh_i dH/dx_i ; gG += gh_i w */
static void size_backward(const unroll_t* U, const double* x, const double* gh, double* lam, double* gG) {
    for (int i = 0; i < U->n; ++i) {
        if (gh[i] == 0.0) continue;
        double g[3], w[8];
        long idx[8];
        size_at(U, x + 3 * i, g, idx, w);
        for (int d = 0; d < 3; ++d) lam[3 * i + d] += gh[i] * g[d];
        for (int k = 0; k < 8; ++k) gG[idx[k]] += gh[i] * w[k];
    }
}

static void loss_backward(const unroll_t* U, const double* x, double* h, double* gh, double* lam, double* gG) {
    memset(gh, 0, sizeof(double) * U->n);
    for (int i = 0; i < U->n; ++i) h[i] = size_at(U, x + 3 * i, NULL, NULL, NULL);
    for (int i = 0; i < U->n; ++i)
        for (int k = 0; k < U->nnb[i]; ++k) {
            int j = U->nbr[(long)i * UK + k];
            double e[3] = { x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2] };
            double l = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            double hm = 0.5 * (h[i] + h[j]);
            double r = l / hm - 1.0;
            double dl = 2.0 * r / hm, dhm = -2.0 * r * l / (hm * hm);
            for (int d = 0; d < 3; ++d) {
                lam[3 * i + d] += dl * e[d] / l;
                lam[3 * j + d] -= dl * e[d] / l;
            }
            gh[i] += 0.5 * dhm;
            gh[j] += 0.5 * dhm;
        }
    size_backward(U, x, gh, lam, gG);
}

/* lam_in: dL/dx_{t+1}; out: lam_out = dL/dx_t (gG accumulated) */
static void step_backward(const unroll_t* U, const double* x, double* h, double* gh, const double* lam_in,
                          double* lam_out, double* gG, const uint32_t* mask) {
    memcpy(lam_out, lam_in, sizeof(double) * 3 * U->n);
    memset(gh, 0, sizeof(double) * U->n);
    for (int i = 0; i < U->n; ++i) h[i] = size_at(U, x + 3 * i, NULL, NULL, NULL);
    for (int i = 0; i < U->n; ++i) {
        if (U->typ[i] == 3) continue;
        int c = __builtin_popcount(mask[i]);
        double mu[3];
        for (int d = 0; d < 3; ++d) mu[d] = U->dt * lam_in[3 * i + d] / (c > 1 ? c : 1);
        project(U, i, mu);
        for (int k = 0; k < U->nnb[i]; ++k) {
            int j = U->nbr[(long)i * UK + k];
            double e[3] = { x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2] };
            double l = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            double a = coef(U, i, j), l0 = a * (h[i] + h[j]);
            if (!((mask[i] >> k) & 1u)) continue;
            double f = (l0 - l) / l, dfl = -l0 / (l * l);
            double em = (e[0] * mu[0] + e[1] * mu[1] + e[2] * mu[2]);
            for (int d = 0; d < 3; ++d) {
                double v = f * mu[d] + e[d] / l * dfl * em;
                lam_out[3 * i + d] += v;
                lam_out[3 * j + d] -= v;
            }
            double s = em / l;
            gh[i] += a * s;
            gh[j] += a * s;
        }
    }
    size_backward(U, x, gh, lam_out, gG);
}

static unroll_t make(int n, const int32_t* nbr, const int32_t* nnb, const uint8_t* typ, const int32_t* m,
                     const double* cs, const double* G, double fscale, double fsurf, double dt) {
    unroll_t U;
    U.n = n;
    U.nbr = nbr;
    U.nnb = nnb;
    U.typ = typ;
    for (int d = 0; d < 3; ++d) {
        U.m[d] = m[d];
        U.cs[d] = cs[d];
    }
    U.G = G;
    U.fscale = fscale;
    U.fsurf = fsurf;
    U.dt = dt;
    U.dirs = NULL;
    return U;
}

/* K steps from x0 (n x 3) into xK; returns the loss at xK. tape: K x n masks,
   recorded (replay = 0) or replayed (replay = 1); dirs: taped constraints or NULL */
double orc_unroll_forward_f64(int n, const int32_t* nbr, const int32_t* nnb, const uint8_t* typ, const int32_t* m,
                              const double* cs, const double* G, double fscale, double fsurf, double dt, int K,
                              const double* x0, double* xK, uint32_t* tape, int replay, const double* dirs) {
    unroll_t U = make(n, nbr, nnb, typ, m, cs, G, fscale, fsurf, dt);
    U.dirs = dirs;
    double* a = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    double* b = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    double* h = (double*)malloc(sizeof(double) * (size_t)n);
    memcpy(a, x0, sizeof(double) * 3 * (size_t)n);
    for (int t = 0; t < K; ++t) {
        step(&U, a, b, h, tape + (size_t)t * n, replay);
        double* s = a;
        a = b;
        b = s;
    }
    memcpy(xK, a, sizeof(double) * 3 * (size_t)n);
    double L = loss_at(&U, a, h);
    free(a);
    free(b);
    free(h);
    return L;
}

/* loss after K steps, and its gradient w.r.t. x0 (n x 3) and G (m0 m1 m2), of
   the function taped by this call's forward pass (replay = 0) or by `tape` */
double orc_unroll_grad_f64(int n, const int32_t* nbr, const int32_t* nnb, const uint8_t* typ, const int32_t* m,
                           const double* cs, const double* G, double fscale, double fsurf, double dt, int K,
                           const double* x0, double* gx0, double* gG, uint32_t* tape, int replay,
                           const double* dirs) {
    unroll_t U = make(n, nbr, nnb, typ, m, cs, G, fscale, fsurf, dt);
    U.dirs = dirs;
    size_t s3 = 3 * (size_t)n;
    double* X = (double*)malloc(sizeof(double) * s3 * (size_t)(K + 1));
    double* h = (double*)malloc(sizeof(double) * (size_t)n);
    double* gh = (double*)malloc(sizeof(double) * (size_t)n);
    double* lam = (double*)calloc(s3, sizeof(double));
    double* lam2 = (double*)calloc(s3, sizeof(double));
    memcpy(X, x0, sizeof(double) * s3);
    for (int t = 0; t < K; ++t) step(&U, X + s3 * t, X + s3 * (t + 1), h, tape + (size_t)t * n, replay);
    double L = loss_at(&U, X + s3 * K, h);
    memset(gG, 0, sizeof(double) * (size_t)m[0] * m[1] * m[2]);
    loss_backward(&U, X + s3 * K, h, gh, lam, gG);
    for (int t = K - 1; t >= 0; --t) {
        step_backward(&U, X + s3 * t, h, gh, lam, lam2, gG, tape + (size_t)t * n);
        double* s = lam;
        lam = lam2;
        lam2 = s;
    }
    memcpy(gx0, lam, sizeof(double) * s3);
    free(X);
    free(h);
    free(gh);
    free(lam);
    free(lam2);
    return L;
}
