/*
 * v2m_oracle.c -- TEST INFRASTRUCTURE ONLY: the plain-C restatement of the
 * relaxation loop (v2m_oracle_body.h) in two precisions, with a C ABI for the
 * Python checkers (oracle/oracle.py):
 *
 *   orc_*_f32   float, compiled without contraction: the reference CPU's arithmetic
 *   orc_*_f64   double: the FP64 checker of forces and positions
 *
 * State arrays are read and written in the variant's own scalar type (float or
 * double); integer arrays are int32 / uint8 / uint16 like the reference's.
 * Nothing in the product links or loads this library.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/v2m_cuda.h"

/* ---- float -------------------------------------------------------------------- */
#define REAL float
#define K(x) x##f
#define FN(name) orcf_##name
#define SQRT sqrtf
#define FLOOR floorf
#define CEIL ceilf
#define FABS fabsf
#define FMIN fminf
#define FMAX fmaxf
#include "v2m_oracle_body.h"
#define POW powf
#include "v2m_seed_oracle_body.h"
#undef POW
#undef REAL
#undef K
#undef FN
#undef SQRT
#undef FLOOR
#undef CEIL
#undef FABS
#undef FMIN
#undef FMAX

/* ---- double ------------------------------------------------------------------- */
#define REAL double
#define K(x) x
#define FN(name) orcd_##name
#define SQRT sqrt
#define FLOOR floor
#define CEIL ceil
#define FABS fabs
#define FMIN fmin
#define FMAX fmax
#include "v2m_oracle_body.h"
#undef REAL
#undef K
#undef FN
#undef SQRT
#undef FLOOR
#undef CEIL
#undef FABS
#undef FMIN
#undef FMAX

/* ---- C ABI -------------------------------------------------------------------- */
#define ORACLE_API(SUF, PFX, REALT)                                                                             \
    void* orc_create_##SUF(const v2m_grid_view* g, const v2m_relax_params* p, const v2m_nodes_view* nd) {      \
        return PFX##create(g, p, nd);                                                                            \
    }                                                                                                            \
    void orc_free_##SUF(void* s) { PFX##free((PFX##state*)s); }                                                \
    int orc_rebuild_##SUF(void* s) {                                                                             \
        PFX##rebuild((PFX##state*)s);                                                                            \
        return 0;                                                                                                \
    }                                                                                                            \
    int orc_force_##SUF(void* s) {                                                                               \
        PFX##force((PFX##state*)s);                                                                              \
        return 0;                                                                                                \
    }                                                                                                            \
    int orc_move_##SUF(void* s) {                                                                                \
        PFX##move_all((PFX##state*)s);                                                                           \
        return 0;                                                                                                \
    }                                                                                                            \
    int orc_tail_##SUF(void* s) { return PFX##tail((PFX##state*)s); }                                           \
    int orc_run_##SUF(void* s) {                                                                                 \
        PFX##state* st = (PFX##state*)s;                                                                         \
        PFX##rebuild(st);                                                                                        \
        for (int it = st->it; it < st->prm.max_iters; ++it) {                                                    \
            PFX##force(st);                                                                                      \
            if (PFX##tail(st)) break;                                                                            \
        }                                                                                                        \
        return 0;                                                                                                \
    }                                                                                                            \
    int orc_info_##SUF(void* s, int64_t* nkeys, int32_t* nlev) {                                                 \
        PFX##state* st = (PFX##state*)s;                                                                         \
        *nkeys = st->nkeys;                                                                                      \
        *nlev = st->nlev;                                                                                        \
        return 0;                                                                                                \
    }                                                                                                            \
    int orc_counts_##SUF(void* s, int32_t* iv, double* dv) {                                                     \
        PFX##state* st = (PFX##state*)s;                                                                         \
        iv[0] = st->it; iv[1] = st->stopped; iv[2] = st->nhalf; iv[3] = st->nrefresh;                            \
        iv[4] = st->rebuilds; iv[5] = st->resets; iv[6] = st->npos; iv[7] = 0;                                   \
        dv[0] = (double)st->fdt; dv[1] = (double)st->falpha; dv[2] = st->power; dv[3] = (double)st->mmax;        \
        dv[4] = (double)st->p99;                                                                                 \
        return 0;                                                                                                \
    }                                                                                                            \
    int64_t orc_read_##SUF(void* s, int what, void* out, int64_t bytes) {                                        \
        PFX##state* st = (PFX##state*)s;                                                                         \
        const void* src = NULL;                                                                                  \
        int64_t nb = 0, n = st->n;                                                                               \
        switch (what) {                                                                                          \
        case V2M_ARR_KEY: src = st->key; nb = 4 * n; break;                                                      \
        case V2M_ARR_SORTED: src = st->sorted; nb = 4 * n; break;                                                \
        case V2M_ARR_CSTART: src = st->cstart; nb = 4 * ((int64_t)st->nkeys + 1); break;                        \
        case V2M_ARR_PS: src = st->Ps; nb = (int64_t)sizeof(REALT) * 4 * n; break;                               \
        case V2M_ARR_NBR: src = st->nbr; nb = 4 * n * V2M_K; break;                                              \
        case V2M_ARR_NNB: src = st->nnb; nb = 4 * n; break;                                                      \
        case V2M_ARR_F: src = st->F; nb = (int64_t)sizeof(REALT) * 4 * n; break;                                 \
        case V2M_ARR_HN: src = st->hn; nb = (int64_t)sizeof(REALT) * n; break;                                   \
        case V2M_ARR_MV: src = st->mv; nb = (int64_t)sizeof(REALT) * n; break;                                   \
        case V2M_ARR_V: src = st->V; nb = (int64_t)sizeof(REALT) * 3 * n; break;                                 \
        case V2M_ARR_PW: src = st->pw; nb = (int64_t)sizeof(REALT) * n; break;                                   \
        case V2M_ARR_P0: src = st->P0; nb = (int64_t)sizeof(REALT) * 3 * n; break;                               \
        case V2M_ARR_P: src = st->P; nb = (int64_t)sizeof(REALT) * 3 * n; break;                                 \
        case V2M_ARR_TYP: src = st->typ; nb = n; break;                                                          \
        case V2M_ARR_PART: src = st->part; nb = 4 * n; break;                                                    \
        case V2M_ARR_HIST: src = st->hist; nb = 4 * 32; break;                                                   \
        case V2M_ARR_DIRS:                                                                                       \
            nb = (int64_t)sizeof(REALT) * 3 * n;                                                                 \
            if (bytes < nb) return -1;                                                                           \
            PFX##constraint_dirs(st, (REALT*)out);                                                               \
            return nb;                                                                                           \
        default: return -1;                                                                                      \
        }                                                                                                        \
        if (bytes < nb) return -1;                                                                               \
        if (nb) memcpy(out, src, (size_t)nb);                                                                    \
        return nb;                                                                                               \
    }                                                                                                            \
    int orc_write_##SUF(void* s, int what, const void* in, int64_t bytes) {                                      \
        PFX##state* st = (PFX##state*)s;                                                                         \
        void* dst = NULL;                                                                                        \
        int64_t nb = 0, n = st->n;                                                                               \
        switch (what) {                                                                                          \
        case V2M_ARR_P: dst = st->P; nb = (int64_t)sizeof(REALT) * 3 * n; break;                                 \
        case V2M_ARR_TYP: dst = st->typ; nb = n; break;                                                          \
        case V2M_ARR_PART: dst = st->part; nb = 4 * n; break;                                                    \
        case V2M_ARR_HN: dst = st->hn; nb = (int64_t)sizeof(REALT) * n; break;                                   \
        case V2M_ARR_V: dst = st->V; nb = (int64_t)sizeof(REALT) * 3 * n; break;                                 \
        case V2M_ARR_F: dst = st->F; nb = (int64_t)sizeof(REALT) * 4 * n; break;                                 \
        case V2M_ARR_NBR: dst = st->nbr; nb = 4 * n * V2M_K; break;                                              \
        case V2M_ARR_NNB: dst = st->nnb; nb = 4 * n; break;                                                      \
        default: return -1;                                                                                      \
        }                                                                                                        \
        if (bytes != nb) return -1;                                                                              \
        if (nb) memcpy(dst, in, (size_t)nb);                                                                     \
        return 0;                                                                                                \
    }

ORACLE_API(f32, orcf_, float)
ORACLE_API(f64, orcd_, double)

/* A whole relaxation in float, written back into the node view (the CPU-baseline "port"). */
int orc_relax_f32(const v2m_grid_view* g, const v2m_relax_params* p, v2m_nodes_view* nd, v2m_relax_stats* out) {
    orcf_state* s = orcf_create(g, p, nd);
    if (!s) return -1;
    orc_run_f32(s);
    memcpy(nd->P, s->P, sizeof(float) * 3 * (size_t)s->n);
    memcpy(nd->typ, s->typ, (size_t)s->n);
    memcpy(nd->part, s->part, 4 * (size_t)s->n);
    if (out) {
        memset(out, 0, sizeof(*out));
        out->iters = s->it;
        out->rebuilds = s->rebuilds;
        out->last_move = s->mmax;
        out->last_p99 = s->p99;
        out->fire_resets = s->resets;
        out->fire_dt = s->fire ? s->fdt : 0.0f;
        for (int i = 0; i < s->n; ++i) {
            out->n_interior += s->typ[i] == V2M_INTERIOR;
            out->n_interface += s->typ[i] == V2M_INTERFACE;
            out->n_junction += s->typ[i] == V2M_JUNCTION;
            out->n_corner += s->typ[i] == V2M_CORNER;
        }
    }
    orcf_free(s);
    return 0;
}

/* tn::seed_cpu restated (v2m_seed_oracle_body.h), in float. Returns the node
   count; the arrays (P 3n, lab n, typ n, part 2n, part3 n) are written when
   cap >= the count. -1 on failure. */
int64_t orc_seed_f32(const v2m_grid_view* g, const v2m_relax_params* p, int64_t cap, float* P, uint16_t* lab,
                     uint8_t* typ, uint16_t* part, uint16_t* part3) {
    if (!g || !p || !g->grade) return -1;
    v2m_nodes_view none;
    memset(&none, 0, sizeof(none));
    orcf_state* s = orcf_create(g, p, &none);
    if (!s) return -1;
    orcf_seeds o;
    int n = orcf_seed(s, g->grade, p, &o);
    if (n >= 0 && cap >= n && n > 0) {
        memcpy(P, o.P, sizeof(float) * 3 * (size_t)n);
        memcpy(lab, o.lab, 2 * (size_t)n);
        memcpy(typ, o.typ, (size_t)n);
        memcpy(part, o.part, 4 * (size_t)n);
        memcpy(part3, o.part3, 2 * (size_t)n);
    }
    orcf_seeds_free(&o);
    orcf_free(s);
    return n;
}
