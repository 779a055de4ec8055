/*
 * v2m_seed_oracle_body.h -- TEST INFRASTRUCTURE ONLY: tn::seed_cpu
 * (src/v2m_particles.cpp:625-726, the junction pass :80-244) restated in plain
 * C over the relaxation restatement's field queries (v2m_oracle_body.h),
 * serial. v2m_oracle.c includes it once, after the float body (REAL = float,
 * no contraction: the reference CPU's arithmetic). Without the shape-feature
 * pass, as the device seeding.
 *
 * Written differently from the reference where the result cannot depend on it:
 * the junction candidates are sorted with qsort on (key, vertex) -- the
 * reference's std::sort comparator is the same total order -- and a lattice
 * node is dropped by a scan of all kept seeds (the reference hashes them in
 * cells of 0.4 hmax and scans 27 cells; a seed within 0.4 h <= 0.4 hmax always
 * lies in those cells, so the dropped set is the same).
 *
 * Needs, besides the body's macros: POW.
 */

/* ---- growable node arrays ---------------------------------------------------------- */
typedef struct {
    int n, cap;
    REAL* P;
    uint16_t *lab, *part, *part3;
    uint8_t* typ;
} FN(seeds);

static int FN(seeds_push)(FN(seeds)* o, const REAL* p, int lab, int typ, int pa, int pb, int pc) {
    if (o->n == o->cap) {
        int c = o->cap ? 2 * o->cap : 1024;
        REAL* P = (REAL*)realloc(o->P, sizeof(REAL) * 3 * (size_t)c);
        uint16_t* L = (uint16_t*)realloc(o->lab, 2 * (size_t)c);
        uint16_t* Q = (uint16_t*)realloc(o->part, 4 * (size_t)c);
        uint16_t* R = (uint16_t*)realloc(o->part3, 2 * (size_t)c);
        uint8_t* T = (uint8_t*)realloc(o->typ, (size_t)c);
        if (P) o->P = P;
        if (L) o->lab = L;
        if (Q) o->part = Q;
        if (R) o->part3 = R;
        if (T) o->typ = T;
        if (!P || !L || !Q || !R || !T) return -1;
        o->cap = c;
    }
    int i = o->n++;
    o->P[3 * i] = p[0];
    o->P[3 * i + 1] = p[1];
    o->P[3 * i + 2] = p[2];
    o->lab[i] = (uint16_t)lab;
    o->typ[i] = (uint8_t)typ;
    o->part[2 * i] = (uint16_t)pa;
    o->part[2 * i + 1] = (uint16_t)pb;
    o->part3[i] = (uint16_t)pc;
    return 0;
}

static void FN(seeds_free)(FN(seeds)* o) {
    free(o->P);
    free(o->lab);
    free(o->part);
    free(o->part3);
    free(o->typ);
    memset(o, 0, sizeof(*o));
}

/* ---- the lattice (src/opencl/v2m_seed_body.cl:424-500) ----------------------------- */
static int FN(seed_level)(int grade, int nseed) {
    return nseed <= 1 ? 0 : (int)FLOOR((REAL)grade * (REAL)(nseed - 1) / K(255.0) + K(0.5));
}

static REAL FN(seed_spacing)(int level, int nseed, REAL hmin, REAL hmax) {
    return nseed <= 1 ? hmin : hmin * POW(hmax / hmin, (REAL)level / (REAL)(nseed - 1));
}

/* the owner label of v2m_label_of, with the voxel mode's answer */
static int FN(label_of)(const FN(state)* s, int voxmode, const REAL* p) {
    int sec;
    if (!voxmode) return FN(owner)(s, p, &sec);
    int lab[V2M_BL];
    if (FN(labels_near)(s, p, lab) == 1) return lab[0];
    int i = (int)FLOOR(p[0] / s->vx + K(0.5)), j = (int)FLOOR(p[1] / s->vy + K(0.5)), k = (int)FLOOR(p[2] / s->vz + K(0.5));
    return FN(label_at)(s, i, j, k);
}

static int FN(seed_voxel)(const FN(state)* s, const uint8_t* grade, int nseed, int voxmode, int i, int j, int k,
                          FN(seeds)* out) {
    size_t v = i + (size_t)s->nx * (j + (size_t)s->ny * k);
    if (s->L[v] == 0) return 0;
    REAL sp = FN(seed_spacing)(FN(seed_level)(grade[v], nseed), nseed, (REAL)s->hmin, (REAL)s->hmax);
    REAL dy = sp * K(0.8660254), dz = sp * K(0.8164966);
    REAL x0 = (i - K(0.5)) * s->vx, x1 = (i + K(0.5)) * s->vx;
    REAL y0 = (j - K(0.5)) * s->vy, y1 = (j + K(0.5)) * s->vy;
    REAL z0 = (k - K(0.5)) * s->vz, z1 = (k + K(0.5)) * s->vz;
    int n = 0;
    int k0 = (int)CEIL(z0 / dz), k1 = (int)CEIL(z1 / dz);
    for (int kk = k0; kk < k1; ++kk) {
        REAL oy = (kk & 1) ? dy / K(3.0) : K(0.0);
        int j0 = (int)CEIL((y0 - oy) / dy), j1 = (int)CEIL((y1 - oy) / dy);
        for (int jj = j0; jj < j1; ++jj) {
            REAL ox = ((jj & 1) ? K(0.5) * sp : K(0.0)) + ((kk & 1) ? K(0.5) * sp : K(0.0));
            int i0 = (int)CEIL((x0 - ox) / sp), i1 = (int)CEIL((x1 - ox) / sp);
            for (int ii = i0; ii < i1; ++ii) {
                REAL p[3];
                p[0] = ii * sp + ((jj & 1) ? K(0.5) * sp : K(0.0)) + ((kk & 1) ? K(0.5) * sp : K(0.0));
                p[1] = jj * dy + ((kk & 1) ? dy / K(3.0) : K(0.0));
                p[2] = kk * dz;
                int l = FN(label_of)(s, voxmode, p);
                if (l == 0 || l == V2M_NOLAB) continue;
                if (FN(seeds_push)(out, p, l, V2M_INTERIOR, V2M_NOLAB, V2M_NOLAB, V2M_NOLAB)) return -1;
                ++n;
            }
        }
    }
    return n;
}

/* src/opencl/v2m_seed_body.cl:509-596 */
static void FN(seed_classify)(const FN(state)* s, FN(seeds)* o, int i) {
    REAL* P = o->P + 3 * (size_t)i;
    REAL p[3] = { P[0], P[1], P[2] };
    o->typ[i] = V2M_INTERIOR;
    o->part[2 * i] = o->part[2 * i + 1] = V2M_NOLAB;
    int a = o->lab[i];
    int nl[V2M_BL];
    int n = FN(labels_near)(s, p, nl);
    if (n < 2) return;
    int b = V2M_NOLAB;
    REAL pb = K(-1.0);
    for (int t = 0; t < n; ++t)
        if (nl[t] != a) {
            REAL v = FN(phi_at)(s, nl[t], p);
            if (v > pb) {
                pb = v;
                b = nl[t];
            }
        }
    if (b == V2M_NOLAB || (b != 0 && b < a)) return;
    int vi = (int)FLOOR(p[0] / s->vx + K(0.5)), vj = (int)FLOOR(p[1] / s->vy + K(0.5)), vk = (int)FLOOR(p[2] / s->vz + K(0.5));
    vi = vi < 0 ? 0 : (vi >= s->nx ? s->nx - 1 : vi);
    vj = vj < 0 ? 0 : (vj >= s->ny ? s->ny - 1 : vj);
    vk = vk < 0 ? 0 : (vk >= s->nz ? s->nz - 1 : vk);
    REAL hs = (REAL)s->hv[vi + (size_t)s->nx * (vj + (size_t)s->ny * vk)];
    REAL g[3];
    REAL v = FN(psi_grad)(s, a, b, p, g);
    REAL gn = SQRT(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (gn < K(1e-9) || FABS(v) / gn > K(0.5) * hs) return;
    REAL q[3] = { p[0], p[1], p[2] };
    if (!FN(project1)(s, a, b, q, K(0.6) * hs)) return;
    o->typ[i] = V2M_INTERFACE;
    o->part[2 * i] = (uint16_t)b;
    int c = V2M_NOLAB;
    REAL pc = K(-1.0), pa = FN(phi_at)(s, a, q);
    for (int t = 0; t < n; ++t)
        if (nl[t] != a && nl[t] != b) {
            REAL w = FN(phi_at)(s, nl[t], q);
            if (w > pc) {
                pc = w;
                c = nl[t];
            }
        }
    if (c != V2M_NOLAB && pc > K(0.5) * pa) {
        REAL r[3] = { q[0], q[1], q[2] };
        if (FN(project2)(s, a, b, c, r, K(0.5) * hs)) {
            q[0] = r[0];
            q[1] = r[1];
            q[2] = r[2];
            o->typ[i] = V2M_JUNCTION;
            o->part[2 * i + 1] = (uint16_t)c;
        }
    }
    P[0] = q[0];
    P[1] = q[1];
    P[2] = q[2];
}

/* ---- grid vertices (src/opencl/v2m_seed_body.cl:611-748) ------------------------------ */
static int FN(vertex_nlab)(const FN(state)* s, int i, int j, int k, int* labs) {
    int n = 0;
    for (int m = 0; m < 8; ++m) {
        int l = FN(label_at)(s, i + (m & 1), j + ((m >> 1) & 1), k + (m >> 2)), seen = 0;
        for (int x = 0; x < n; ++x) seen |= labs[x] == l;
        if (!seen) labs[n++] = l;
    }
    return n;
}

static REAL FN(det3)(REAL M[3][3]) {
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

static int FN(corner_vertex)(const FN(state)* s, int i, int j, int k, FN(seeds)* out) {
    int labs[8];
    int n = FN(vertex_nlab)(s, i, j, k, labs);
    if (n < 4) return 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                if (dz < 0 || (dz == 0 && (dy < 0 || (dy == 0 && dx < 0)))) {
                    int l2[8];
                    if (FN(vertex_nlab)(s, i + dx, j + dy, k + dz, l2) >= 4) return 0;
                }
    REAL x[3] = { (i + K(0.5)) * s->vx, (j + K(0.5)) * s->vy, (k + K(0.5)) * s->vz };
    REAL ph[8];
    for (int t = 0; t < n; ++t) ph[t] = FN(phi_at)(s, labs[t], x);
    for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b)
            if (ph[b] > ph[a]) {
                REAL f = ph[a];
                ph[a] = ph[b];
                ph[b] = f;
                int l = labs[a];
                labs[a] = labs[b];
                labs[b] = l;
            }
    int ia = 0;
    while (ia < 4 && labs[ia] == 0) ++ia;
    int a = labs[ia], o[3], no = 0;
    for (int t = 0; t < 4; ++t)
        if (t != ia) o[no++] = labs[t];
    REAL q[3] = { x[0], x[1], x[2] };
    int ok = 1;
    for (int it = 0; it < 5 && ok; ++it) {
        REAL J[3][3], v[3];
        for (int r = 0; r < 3; ++r) v[r] = FN(psi_grad)(s, a, o[r], q, J[r]);
        REAL det = FN(det3)(J);
        if (FABS(det) < K(1e-12)) {
            ok = 0;
            break;
        }
        REAL dlt[3];
        for (int c = 0; c < 3; ++c) {
            REAL M[3][3];
            for (int r = 0; r < 3; ++r)
                for (int cc = 0; cc < 3; ++cc) M[r][cc] = cc == c ? -v[r] : J[r][cc];
            dlt[c] = FN(det3)(M) / det;
        }
        for (int c = 0; c < 3; ++c) q[c] += dlt[c];
    }
    REAL ex = (q[0] - x[0]) / s->vx, ey = (q[1] - x[1]) / s->vy, ez = (q[2] - x[2]) / s->vz;
    if (ok && ex * ex + ey * ey + ez * ez <= K(0.25)) {
        x[0] = q[0];
        x[1] = q[1];
        x[2] = q[2];
    }
    return FN(seeds_push)(out, x, a, V2M_CORNER, o[0], o[1], o[2]) ? -1 : 1;
}

/* a junction-line candidate (src/opencl/v2m_particle_body.cl:302-356) */
typedef struct {
    int key[7];
    int64_t vert;
    REAL x[3];
    int lab3[3];
} FN(jcand);

static int FN(jcand_cmp)(const void* pa, const void* pb) {
    const FN(jcand)* p = (const FN(jcand)*)pa;
    const FN(jcand)* q = (const FN(jcand)*)pb;
    for (int e = 0; e < 7; ++e)
        if (p->key[e] != q->key[e]) return p->key[e] < q->key[e] ? -1 : 1;
    return p->vert < q->vert ? -1 : (p->vert > q->vert ? 1 : 0);
}

static int FN(junction_vertex)(const FN(state)* s, const uint8_t* grade, int nseed, REAL cellfac, int i, int j, int k,
                               FN(jcand)* c) {
    int labs[8];
    if (FN(vertex_nlab)(s, i, j, k, labs) != 3) return 0;
    REAL* x = c->x;
    x[0] = (i + K(0.5)) * s->vx;
    x[1] = (j + K(0.5)) * s->vy;
    x[2] = (k + K(0.5)) * s->vz;
    int a = -1;
    REAL pa = K(-1.0);
    for (int t = 0; t < 3; ++t)
        if (labs[t] != 0) {
            REAL f = FN(phi_at)(s, labs[t], x);
            if (f > pa) {
                pa = f;
                a = labs[t];
            }
        }
    int o[2], no = 0;
    for (int t = 0; t < 3; ++t)
        if (labs[t] != a) o[no++] = labs[t];
    REAL vmin = FMIN(FMIN(s->vx, s->vy), s->vz);
    if (!FN(project2)(s, a, o[0], o[1], x, vmin) || !FN(valid_on)(s, a, o[0], o[1], x)) return 0;
    int vi = (int)FLOOR(x[0] / s->vx + K(0.5)), vj = (int)FLOOR(x[1] / s->vy + K(0.5)), vk = (int)FLOOR(x[2] / s->vz + K(0.5));
    if (vi < 0 || vj < 0 || vk < 0 || vi >= s->nx || vj >= s->ny || vk >= s->nz) return 0;
    int lev = FN(seed_level)(grade[vi + (size_t)s->nx * (vj + (size_t)s->ny * vk)], nseed);
    REAL cc = cellfac * FN(seed_spacing)(lev, nseed, (REAL)s->hmin, (REAL)s->hmax);
    c->lab3[0] = a;
    c->lab3[1] = o[0];
    c->lab3[2] = o[1];
    int t[3] = { a, o[0], o[1] };
    for (int u = 0; u < 2; ++u)
        for (int w = 0; w < 2 - u; ++w)
            if (t[w] > t[w + 1]) {
                int z = t[w];
                t[w] = t[w + 1];
                t[w + 1] = z;
            }
    c->key[0] = lev;
    c->key[1] = (int)FLOOR(x[0] / cc);
    c->key[2] = (int)FLOOR(x[1] / cc);
    c->key[3] = (int)FLOOR(x[2] / cc);
    c->key[4] = t[0];
    c->key[5] = t[1];
    c->key[6] = t[2];
    return 1;
}

/* the whole seeding; returns the node count, -1 on allocation failure */
static int FN(seed)(const FN(state)* s, const uint8_t* grade, const v2m_relax_params* prm, FN(seeds)* out) {
    memset(out, 0, sizeof(*out));
    int voxmode = prm->voxel_trap != 0;
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i)
                if (FN(seed_voxel)(s, grade, prm->nseed, voxmode, i, j, k, out) < 0) return -1;
    for (int i = 0; i < out->n; ++i) FN(seed_classify)(s, out, i);
    int vx1 = s->nx + 1, vy1 = s->ny + 1, vz1 = s->nz + 1;
    int64_t nvert = (int64_t)vx1 * vy1 * vz1;
    if (prm->jseed > 0.0f) {
        int m = 0, cap = 0;
        FN(jcand)* cand = NULL;
        for (int64_t v = 0; v < nvert; ++v) {
            int i = (int)(v % vx1) - 1, j = (int)((v / vx1) % vy1) - 1, k = (int)(v / ((int64_t)vx1 * vy1)) - 1;
            FN(jcand) c;
            if (!FN(junction_vertex)(s, grade, prm->nseed, (REAL)prm->jseed, i, j, k, &c)) continue;
            c.vert = v;
            if (m == cap) {
                cap = cap ? 2 * cap : 256;
                FN(jcand)* nc = (FN(jcand)*)realloc(cand, sizeof(FN(jcand)) * (size_t)cap);
                if (!nc) {
                    free(cand);
                    return -1;
                }
                cand = nc;
            }
            cand[m++] = c;
        }
        if (m > 1) qsort(cand, (size_t)m, sizeof(FN(jcand)), FN(jcand_cmp));
        int ns = 0;   /* the kept seeds, compacted to the front */
        for (int e = 0; e < m; ++e)
            if (e == 0 || memcmp(cand[e].key, cand[e - 1].key, sizeof(cand[e].key)) != 0) cand[ns++] = cand[e];
        FN(seeds) kept;
        memset(&kept, 0, sizeof(kept));
        int fail = 0;
        for (int i = 0; i < out->n && !fail; ++i) {
            const REAL* p = out->P + 3 * (size_t)i;
            int drop = 0;
            if (out->typ[i] != V2M_CORNER) {
                /* h at the nearest voxel (v2m_h_at), whatever the relaxation's h mode */
                int hi = (int)FLOOR(p[0] / s->vx + K(0.5)), hj = (int)FLOOR(p[1] / s->vy + K(0.5)),
                    hk = (int)FLOOR(p[2] / s->vz + K(0.5));
                hi = hi < 0 ? 0 : (hi >= s->nx ? s->nx - 1 : hi);
                hj = hj < 0 ? 0 : (hj >= s->ny ? s->ny - 1 : hj);
                hk = hk < 0 ? 0 : (hk >= s->nz ? s->nz - 1 : hk);
                REAL h = (REAL)s->hv[hi + (size_t)s->nx * (hj + (size_t)s->ny * hk)];
                for (int e = 0; e < ns && !drop; ++e) {
                    REAL ex = p[0] - cand[e].x[0], ey = p[1] - cand[e].x[1], ez = p[2] - cand[e].x[2];
                    drop = ex * ex + ey * ey + ez * ez < K(0.16) * h * h;
                }
            }
            if (!drop)
                fail = FN(seeds_push)(&kept, p, out->lab[i], out->typ[i], out->part[2 * i], out->part[2 * i + 1],
                                      out->part3[i]);
        }
        for (int e = 0; e < ns && !fail; ++e)
            fail = FN(seeds_push)(&kept, cand[e].x, cand[e].lab3[0], V2M_JUNCTION, cand[e].lab3[1], cand[e].lab3[2],
                                  V2M_NOLAB);
        free(cand);
        FN(seeds_free)(out);
        *out = kept;
        if (fail) return -1;
    }
    if (prm->corners) {
        for (int64_t v = 0; v < nvert; ++v) {
            int i = (int)(v % vx1) - 1, j = (int)((v / vx1) % vy1) - 1, k = (int)(v / ((int64_t)vx1 * vy1)) - 1;
            if (FN(corner_vertex)(s, i, j, k, out) < 0) return -1;
        }
    }
    return out->n;
}
