/*
 * v2m_oracle_body.h -- TEST INFRASTRUCTURE ONLY: the relaxation restated in
 * plain C, serial, over one scalar type. v2m_oracle.c includes it twice: REAL =
 * float (compiled with -ffp-contract=off: the reference CPU's arithmetic) and
 * REAL = double (the FP64 checker of the float paths). Only tests, the smoke
 * check and the CPU-baseline leg of the benchmark use it.
 *
 * Each function names the fangq/trussnet code it restates. The K-nearest lists
 * are built differently from the reference (every accepted candidate collected,
 * then sorted by (distance, id) and cut at K), which gives the same lists
 * because the reference's insertion keeps exactly the K smallest in that total
 * order (src/opencl/v2m_particle_body.cl:127-141).
 *
 * Needs, before inclusion: REAL, K(x) (a literal of type REAL), FN(name),
 * SQRT, FLOOR, CEIL, FABS, FMIN, FMAX.
 */

/* ---- state ------------------------------------------------------------------- */
typedef struct {
    /* grid (caller memory, float) */
    int nx, ny, nz, nbx, nby, nbz;
    REAL vx, vy, vz;
    const uint16_t* L;
    const int32_t* bl_cnt;
    const uint16_t* bl_lab;
    const int32_t* bl_slot;
    const float* phi;
    const float* hv;
    const float* gI;
    const float* gTW;
    int gm;
    int64_t ntw;            /* floats in gTW (the analytic shape program when gm < 0) */
    float hmin, hmax;
    /* parameters */
    v2m_relax_params prm;
    int fire, voxmode, hmode, rebuild_div;
    /* hash (src/opencl/v2m_particle_body.cl:21-27) */
    REAL b0, ox, oy, oz;
    int nlev, dim[V2M_MAXLEV][3], off[V2M_MAXLEV], nkeys;
    /* nodes */
    int n;
    REAL *P, *P0, *hn, *F, *V, *pw, *mv, *Ps;
    uint16_t* lab;
    uint8_t* typ;
    uint16_t* part;
    int *key, *cstart, *sorted, *nbr, *nnb;
    /* loop */
    REAL fdt, fdt0, fdtmax, falpha;
    int npos, resets, it, stopped, rebuilds, nhalf, nrefresh, hist[32];
    REAL mmax, p99;
    double power;
} FN(state);

/* ---- grid lookups (src/opencl/v2m_grid_body.cl:71-200) ----------------------- */
static int FN(label_at)(const FN(state)* s, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= s->nx || j >= s->ny || k >= s->nz) return 0;
    return s->L[i + (size_t)s->nx * (j + (size_t)s->ny * k)];
}

static int FN(brick)(const FN(state)* s, int i, int j, int k) {
    return (i >> 3) + s->nbx * ((j >> 3) + s->nby * (k >> 3));
}

static int FN(slot)(const FN(state)* s, int b, int l, int* has) {
    int c = s->bl_cnt[b];
    *has = 0;
    for (int q = 0; q < c && q < V2M_BL; ++q) {
        if (s->bl_lab[(size_t)b * V2M_BL + q] == l) {
            *has = 1;
            return s->bl_slot[b] < 0 ? -1 : s->bl_slot[b] + q;
        }
    }
    return -1;
}

static REAL FN(phi_vox)(const FN(state)* s, int l, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= s->nx || j >= s->ny || k >= s->nz) return l == 0 ? K(1.0) : K(0.0);
    int has;
    int sl = FN(slot)(s, FN(brick)(s, i, j, k), l, &has);
    if (sl < 0) return (has && s->L[i + (size_t)s->nx * (j + (size_t)s->ny * k)] == l) ? K(1.0) : K(0.0);
    return (REAL)s->phi[(size_t)sl * V2M_SLOT + (i & 7) + 8 * ((j & 7) + 8 * (k & 7))];
}

/* corner c of the cell at (i0,j0,k0): bit 0 +i, bit 1 +j, bit 2 +k. The
   reference fetches a single-brick cell's slot once (v2m_phi_cell); the values
   are the same as corner by corner. */
static void FN(cell)(const FN(state)* s, int l, int i0, int j0, int k0, REAL* c) {
    for (int m = 0; m < 8; ++m) c[m] = FN(phi_vox)(s, l, i0 + (m & 1), j0 + ((m >> 1) & 1), k0 + ((m >> 2) & 1));
}

static REAL FN(blend)(const REAL* c, REAL fx, REAL fy, REAL fz) {
    REAL x00 = c[0] + fx * (c[1] - c[0]), x10 = c[2] + fx * (c[3] - c[2]);
    REAL x01 = c[4] + fx * (c[5] - c[4]), x11 = c[6] + fx * (c[7] - c[6]);
    REAL y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    return y0 + fz * (y1 - y0);
}

/* ---- analytic shape fields, gm < 0 (src/opencl/v2m_sdf_body.cl:75-478) -------------
 * One postfix program per label over nine primitive types, min / max with the
 * crease blend and the gap closing, complement, sums and scales, bounding-box
 * culling and per-brick programs; a values-only pass, then one with the
 * gradients (central differences of each primitive) only where a min / max
 * needs them. Every program read is bounds-checked. */
typedef struct {
    REAL v, x, y, z;
} FN(sv);

static REAL FN(pg)(const FN(state)* s, int64_t k) {
    return (k >= 0 && k < s->ntw) ? (REAL)s->gTW[k] : K(0.0);
}

static int FN(sdf_np)(int t) {
    switch (t) {
    case 1: return 4;
    case 2: case 4: return 6;
    case 3: case 9: return 7;
    case 5: case 6: case 8: return 8;
    case 7: return 15;
    default: return 0;
    }
}

static REAL FN(sdf_prim)(int t, const float* q, REAL x, REAL y, REAL z) {
    if (t == 1) { /* sphere c r */
        REAL dx = x - q[0], dy = y - q[1], dz = z - q[2];
        return q[3] - SQRT(dx * dx + dy * dy + dz * dz);
    }
    if (t == 2) { /* box lo hi */
        REAL cx = K(0.5) * (q[0] + q[3]), cy = K(0.5) * (q[1] + q[4]), cz = K(0.5) * (q[2] + q[5]);
        REAL ux = FABS(x - cx) - K(0.5) * FABS(q[3] - q[0]), uy = FABS(y - cy) - K(0.5) * FABS(q[4] - q[1]),
             uz = FABS(z - cz) - K(0.5) * FABS(q[5] - q[2]);
        REAL ox = FMAX(ux, K(0.0)), oy = FMAX(uy, K(0.0)), oz = FMAX(uz, K(0.0));
        REAL out = SQRT(ox * ox + oy * oy + oz * oz), in = FMIN(FMAX(ux, FMAX(uy, uz)), K(0.0));
        return -(out + in);
    }
    if (t == 4) return -((x - q[0]) * q[3] + (y - q[1]) * q[4] + (z - q[2]) * q[5]); /* half-space */
    if (t == 5) { /* slab */
        REAL tt = (x - q[0]) * q[3] + (y - q[1]) * q[4] + (z - q[2]) * q[5];
        return FMIN(tt - q[6], q[7] - tt);
    }
    if (t == 9) { /* infinite cylinder */
        REAL dx = x - q[0], dy = y - q[1], dz = z - q[2];
        REAL tt = dx * q[3] + dy * q[4] + dz * q[5];
        REAL rx = dx - tt * q[3], ry = dy - tt * q[4], rz = dz - tt * q[5];
        return q[6] - SQRT(rx * rx + ry * ry + rz * rz);
    }
    if (t == 6) { /* torus */
        REAL dx = x - q[0], dy = y - q[1], dz = z - q[2];
        REAL h = dx * q[3] + dy * q[4] + dz * q[5];
        REAL rx = dx - h * q[3], ry = dy - h * q[4], rz = dz - h * q[5];
        REAL a = SQRT(rx * rx + ry * ry + rz * rz) - q[6];
        return q[7] - SQRT(a * a + h * h);
    }
    if (t == 3) { /* capped cylinder */
        REAL bx = q[3] - q[0], by = q[4] - q[1], bz = q[5] - q[2];
        REAL px = x - q[0], py = y - q[1], pz = z - q[2];
        REAL baba = bx * bx + by * by + bz * bz, paba = px * bx + py * by + pz * bz;
        REAL ex = px * baba - bx * paba, ey = py * baba - by * paba, ez = pz * baba - bz * paba;
        REAL u = SQRT(ex * ex + ey * ey + ez * ez) - q[6] * baba;
        REAL v = FABS(paba - baba * K(0.5)) - baba * K(0.5);
        REAL u2 = u * u, v2 = v * v * baba;
        REAL dd = FMAX(u, v) < K(0.0) ? -FMIN(u2, v2) : ((u > K(0.0) ? u2 : K(0.0)) + (v > K(0.0) ? v2 : K(0.0)));
        return -(dd < K(0.0) ? K(-1.0) : K(1.0)) * SQRT(FABS(dd)) / baba;
    }
    if (t == 8) { /* capped frustum */
        REAL bx = q[3] - q[0], by = q[4] - q[1], bz = q[5] - q[2];
        REAL px = x - q[0], py = y - q[1], pz = z - q[2];
        REAL ra = q[6], rb = q[7];
        REAL rba = rb - ra, baba = bx * bx + by * by + bz * bz;
        REAL papa = px * px + py * py + pz * pz, paba = (px * bx + py * by + pz * bz) / baba;
        REAL xr = SQRT(FMAX(papa - paba * paba * baba, K(0.0)));
        REAL cax = FMAX(K(0.0), xr - ((paba < K(0.5)) ? ra : rb)), cay = FABS(paba - K(0.5)) - K(0.5);
        REAL k = rba * rba + baba;
        REAL f = FMIN(FMAX((rba * (xr - ra) + paba * baba) / k, K(0.0)), K(1.0));
        REAL cbx = xr - ra - f * rba, cby = paba - f;
        REAL sg = (cbx < K(0.0) && cay < K(0.0)) ? K(-1.0) : K(1.0);
        REAL d2 = FMIN(cax * cax + cay * cay * baba, cbx * cbx + cby * cby * baba);
        return -sg * SQRT(d2);
    }
    if (t == 7) { /* ellipsoid bound */
        REAL dx = x - q[0], dy = y - q[1], dz = z - q[2];
        REAL lx = q[6] * dx + q[7] * dy + q[8] * dz, ly = q[9] * dx + q[10] * dy + q[11] * dz,
             lz = q[12] * dx + q[13] * dy + q[14] * dz;
        REAL ax = lx / q[3], ay = ly / q[4], az = lz / q[5];
        REAL bx = ax / q[3], by = ay / q[4], bz = az / q[5];
        REAL k0 = SQRT(ax * ax + ay * ay + az * az), k1 = SQRT(bx * bx + by * by + bz * bz);
        if (k1 < K(1e-20)) return FMIN((REAL)q[3], FMIN((REAL)q[4], (REAL)q[5]));
        return -k0 * (k0 - K(1.0)) / k1;
    }
    return K(-1e30);
}

static FN(sv) FN(sdf_minmax)(FN(sv) a, FN(sv) b, REAL sgn, REAL k, REAL kgap, int grad, int* near) {
    REAL va = sgn * a.v, vb = sgn * b.v;
    int sliver = kgap > K(0.0) && va > -kgap && vb > -kgap && va + vb < kgap;
    if (sliver && !grad) *near = 1;
    REAL pen = K(0.0), dpen = K(0.0);
    if (sliver && grad) {
        REAL ga = SQRT(a.x * a.x + a.y * a.y + a.z * a.z), gb = SQRT(b.x * b.x + b.y * b.y + b.z * b.z);
        if (ga > K(0.0) && gb > K(0.0)) {
            REAL c = (a.x * b.x + a.y * b.y + a.z * b.z) / (ga * gb);
            REAL wg = FMIN(K(1.0), FMAX(K(0.0), (-c - K(0.7)) / K(0.25)));
            REAL u = FMAX(K(0.0), K(1.0) - (va + vb) / kgap);
            pen = kgap * wg * u * u;
            dpen = K(2.0) * wg * u;
        }
    }
    FN(sv) r = a;
    if (k > K(0.0) && FABS(va - vb) < k) {
        if (!grad) {
            *near = 1;
        } else {
            REAL ga = SQRT(a.x * a.x + a.y * a.y + a.z * a.z), gb = SQRT(b.x * b.x + b.y * b.y + b.z * b.z);
            REAL c = ga > K(0.0) && gb > K(0.0) ? (a.x * b.x + a.y * b.y + a.z * b.z) / (ga * gb) : K(0.0);
            k *= FMIN(K(1.0), FMAX(K(0.0), (K(0.995) - c) / K(0.095)));
        }
    }
    if (k > K(0.0) && FABS(va - vb) < k) {
        REAL h = K(0.5) + K(0.5) * (vb - va) / k;
        r.v = sgn * (vb * (K(1.0) - h) + va * h - k * h * (K(1.0) - h));
        r.x = h * a.x + (K(1.0) - h) * b.x;
        r.y = h * a.y + (K(1.0) - h) * b.y;
        r.z = h * a.z + (K(1.0) - h) * b.z;
    } else if (vb < va) {
        r = b;
    }
    r.v -= sgn * pen;
    if (dpen > K(0.0)) {
        r.x += dpen * (a.x + b.x);
        r.y += dpen * (a.y + b.y);
        r.z += dpen * (a.z + b.z);
    }
    return r;
}

static int FN(is_mm)(int op) {
    return op == 2 || op == 3 || op == 10 || op == 11;
}

/* s_l at grid-mm point p, and (wantg) its gradient */
static FN(sv) FN(sdf)(const FN(state)* s, int l, const REAL* p, int wantg) {
    const FN(sv) zero = { K(0.0), K(0.0), K(0.0), K(0.0) };
    FN(sv) none = zero;
    none.v = K(-1e30);
    int N = (int)FN(pg)(s, 0);
    if (l < 0 || l >= N) return none;
    REAL x = p[0] + FN(pg)(s, 2), y = p[1] + FN(pg)(s, 3), z = p[2] + FN(pg)(s, 4);
    int start = (int)FN(pg)(s, 5 + l);
    int T = (int)FN(pg)(s, 8 + N);
    if (T > 0) {
        int nbx = (int)FN(pg)(s, T), nby = (int)FN(pg)(s, T + 1), nbz = (int)FN(pg)(s, T + 2);
        REAL vx = FN(pg)(s, T + 3);
        int bi = (int)FLOOR(p[0] / vx + K(0.5)) >> 3, bj = (int)FLOOR(p[1] / vx + K(0.5)) >> 3,
            bk = (int)FLOOR(p[2] / vx + K(0.5)) >> 3;
        bi = bi < 0 ? 0 : (bi >= nbx ? nbx - 1 : bi);
        bj = bj < 0 ? 0 : (bj >= nby ? nby - 1 : bj);
        bk = bk < 0 ? 0 : (bk >= nbz ? nbz - 1 : bk);
        int64_t e = (int64_t)T + 4 + bi + (int64_t)nbx * (bj + (int64_t)nby * bk);
        start = (int)FN(pg)(s, (int64_t)(int)FN(pg)(s, e) + l);
    }
    REAL kblend = FN(pg)(s, 5 + N), kgap = FN(pg)(s, 6 + N), m = FN(pg)(s, 7 + N);
    FN(sv) st[12];
    int sp = 0, grad = wantg != 0;
    for (int pass = 0; pass < 2; ++pass) {
        int pc = start, near = 0;
        sp = 0;
        for (int guard = 0; guard < 100000; ++guard) {
            int op = (int)FN(pg)(s, pc);
            if (op == 0) break;
            if (FN(is_mm)(op)) {
                if (sp > 1) {
                    st[sp - 2] = FN(sdf_minmax)(st[sp - 2], st[sp - 1], op == 2 || op == 10 ? K(-1.0) : K(1.0), kblend,
                                                op >= 10 ? K(0.0) : kgap, grad, &near);
                    --sp;
                }
                pc += 1;
                continue;
            }
            if (op == 4) {
                if (sp > 0) {
                    st[sp - 1].v = -st[sp - 1].v;
                    st[sp - 1].x = -st[sp - 1].x;
                    st[sp - 1].y = -st[sp - 1].y;
                    st[sp - 1].z = -st[sp - 1].z;
                }
                pc += 1;
                continue;
            }
            if (op == 8) {
                if (sp > 1) {
                    FN(sv) t0 = st[sp - 1], t1 = st[sp - 2];
                    t0.v += t1.v;
                    t0.x += t1.x;
                    t0.y += t1.y;
                    t0.z += t1.z;
                    st[sp - 2] = t0;
                    --sp;
                }
                pc += 1;
                continue;
            }
            if (op == 9) {
                REAL f = FN(pg)(s, pc + 1);
                if (sp > 0) {
                    st[sp - 1].v *= f;
                    st[sp - 1].x *= f;
                    st[sp - 1].y *= f;
                    st[sp - 1].z *= f;
                }
                pc += 2;
                continue;
            }
            FN(sv) nv = zero;
            if (op == 1) {
                int type = (int)FN(pg)(s, pc + 1), np = FN(sdf_np)(type);
                if ((int64_t)pc + 2 + np > s->ntw) break;
                const float* q = s->gTW + pc + 2;
                REAL e = FMAX(K(1e-4) * (FABS((REAL)q[0]) + FABS((REAL)q[1]) + FABS((REAL)q[2]) + K(1.0)), K(1e-5));
                int ne = grad ? 7 : 1;
                REAL fv[7];
                for (int k = 0; k < ne; ++k) {
                    REAL dd = k == 0 ? K(0.0) : ((k & 1) ? e : -e);
                    int ax = (k - 1) >> 1;
                    fv[k] = FN(sdf_prim)(type, q, x + (ax == 0 ? dd : K(0.0)), y + (ax == 1 ? dd : K(0.0)),
                                         z + (ax == 2 ? dd : K(0.0)));
                }
                nv.v = fv[0];
                if (grad) {
                    nv.x = (fv[1] - fv[2]) / (K(2.0) * e);
                    nv.y = (fv[3] - fv[4]) / (K(2.0) * e);
                    nv.z = (fv[5] - fv[6]) / (K(2.0) * e);
                }
                pc += 2 + np;
            } else if (op == 6) {
                if (!(x < FN(pg)(s, pc + 1) - m || y < FN(pg)(s, pc + 2) - m || z < FN(pg)(s, pc + 3) - m ||
                      x > FN(pg)(s, pc + 4) + m || y > FN(pg)(s, pc + 5) + m || z > FN(pg)(s, pc + 6) + m)) {
                    pc += 9;
                    continue;
                }
                nv.v = FN(pg)(s, pc + 8) * m;
                pc += 9 + (int)FN(pg)(s, pc + 7);
            } else if (op == 7) {
                nv.v = FN(pg)(s, pc + 1) * m;
                pc += 2;
            } else if (op == 5) {
                nv.v = FN(pg)(s, pc + 1);
                pc += 2;
            } else {
                break;
            }
            {
                int op1 = (int)FN(pg)(s, pc), neg = op1 == 4;
                int op2 = neg ? (int)FN(pg)(s, pc + 1) : op1;
                if (sp > 0 && FN(is_mm)(op2)) {
                    if (neg) {
                        nv.v = -nv.v;
                        nv.x = -nv.x;
                        nv.y = -nv.y;
                        nv.z = -nv.z;
                    }
                    st[sp - 1] = FN(sdf_minmax)(st[sp - 1], nv, op2 == 2 || op2 == 10 ? K(-1.0) : K(1.0), kblend,
                                                op2 >= 10 ? K(0.0) : kgap, grad, &near);
                    pc += 1 + neg;
                    continue;
                }
            }
            if (sp < 12) st[sp++] = nv;
        }
        if (grad || !near) break;
        grad = 1;
    }
    return sp > 0 ? st[sp - 1] : none;
}

static REAL FN(phi_at)(const FN(state)* s, int l, const REAL* p) {
    if (s->gm < 0) {
        return FMIN(K(1.0), FMAX(K(0.0), K(0.5) + FN(sdf)(s, l, p, 0).v / (REAL)s->gTW[1]));
    }
    REAL u = p[0] / s->vx, v = p[1] / s->vy, w = p[2] / s->vz;
    int i0 = (int)FLOOR(u), j0 = (int)FLOOR(v), k0 = (int)FLOOR(w);
    REAL c[8];
    FN(cell)(s, l, i0, j0, k0, c);
    return FN(blend)(c, u - i0, v - j0, w - k0);
}

/* src/opencl/v2m_seed_body.cl:42-59 */
static int FN(labels_near)(const FN(state)* s, const REAL* p, int* out) {
    int i = (int)FLOOR(p[0] / s->vx + K(0.5)), j = (int)FLOOR(p[1] / s->vy + K(0.5)), k = (int)FLOOR(p[2] / s->vz + K(0.5));
    if (i < 0 || j < 0 || k < 0 || i >= s->nx || j >= s->ny || k >= s->nz) {
        out[0] = 0;
        return 1;
    }
    int b = FN(brick)(s, i, j, k);
    int c = s->bl_cnt[b] < V2M_BL ? s->bl_cnt[b] : V2M_BL;
    for (int q = 0; q < c; ++q) out[q] = s->bl_lab[(size_t)b * V2M_BL + q];
    return c;
}

/* gray-scale intensity and gradient (src/opencl/v2m_seed_body.cl:65-92) */
static REAL FN(gray)(const FN(state)* s, const REAL* p, REAL* g) {
    REAL u = p[0] / s->vx, v = p[1] / s->vy, w = p[2] / s->vz;
    int i0 = (int)FLOOR(u), j0 = (int)FLOOR(v), k0 = (int)FLOOR(w);
    REAL fx = u - i0, fy = v - j0, fz = w - k0;
    REAL outside = (REAL)s->gTW[0] - (REAL)s->gTW[s->gm];
    REAL c[8];
    for (int m = 0; m < 8; ++m) {
        int ii = i0 + (m & 1), jj = j0 + ((m >> 1) & 1), kk = k0 + ((m >> 2) & 1);
        c[m] = (ii < 0 || jj < 0 || kk < 0 || ii >= s->nx || jj >= s->ny || kk >= s->nz)
                   ? outside : (REAL)s->gI[ii + (size_t)s->nx * (jj + (size_t)s->ny * kk)];
    }
    REAL x00 = c[0] + fx * (c[1] - c[0]), x10 = c[2] + fx * (c[3] - c[2]);
    REAL x01 = c[4] + fx * (c[5] - c[4]), x11 = c[6] + fx * (c[7] - c[6]);
    REAL y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    if (g) {
        REAL dx0 = (c[1] - c[0]) + fy * ((c[3] - c[2]) - (c[1] - c[0]));
        REAL dx1 = (c[5] - c[4]) + fy * ((c[7] - c[6]) - (c[5] - c[4]));
        g[0] = (dx0 + fz * (dx1 - dx0)) / s->vx;
        g[1] = ((x10 - x00) + fz * ((x11 - x01) - (x10 - x00))) / s->vy;
        g[2] = (y1 - y0) / s->vz;
    }
    return y0 + fz * (y1 - y0);
}

static int FN(gray_psi)(const FN(state)* s, int a, int b, const REAL* p, REAL* val, REAL* g) {
    if (s->gm < 0) { /* analytic shape fields: (s_a - s_b) / w */
        REAL w = (REAL)s->gTW[1];
        if (!g) {
            *val = (FN(sdf)(s, a, p, 0).v - FN(sdf)(s, b, p, 0).v) / w;
            return 1;
        }
        FN(sv) sa = FN(sdf)(s, a, p, 1), sb = FN(sdf)(s, b, p, 1);
        g[0] = (sa.x - sb.x) / w;
        g[1] = (sa.y - sb.y) / w;
        g[2] = (sa.z - sb.z) / w;
        *val = (sa.v - sb.v) / w;
        return 1;
    }
    if (s->gm <= 0 || (a - b != 1 && b - a != 1)) return 0;
    int k = a < b ? a : b;
    REAL sg = (a > b ? K(2.0) : K(-2.0)) / (REAL)s->gTW[s->gm + k];
    *val = sg * (FN(gray)(s, p, g) - (REAL)s->gTW[k]);
    if (g) {
        g[0] *= sg;
        g[1] *= sg;
        g[2] *= sg;
    }
    return 1;
}

/* owner label (src/opencl/v2m_seed_body.cl:116-175), smooth mode */
static int FN(owner)(const FN(state)* s, const REAL* p, int* second) {
    if (s->gm > 0) {
        REAL I = FN(gray)(s, p, NULL);
        int l = 0;
        while (l < s->gm && I >= (REAL)s->gTW[l]) ++l;
        REAL dl = l > 0 ? (I - (REAL)s->gTW[l - 1]) / (REAL)s->gTW[s->gm + l - 1] : K(1e30);
        REAL du = l < s->gm ? ((REAL)s->gTW[l] - I) / (REAL)s->gTW[s->gm + l] : K(1e30);
        *second = (dl < du) ? l - 1 : (l < s->gm ? l + 1 : V2M_NOLAB);
        return l;
    }
    int lab[V2M_BL];
    int n = FN(labels_near)(s, p, lab);
    int best = lab[0], sec = V2M_NOLAB;
    REAL pb = s->gm < 0 ? K(-1e30) : K(-1.0), ps = pb;
    if (n == 1) {
        *second = V2M_NOLAB;
        return best;
    }
    for (int q = 0; q < n; ++q) {
        /* (analytic fields: ranked by s itself) */
        REAL v = s->gm < 0 ? FN(sdf)(s, lab[q], p, 0).v : FN(phi_at)(s, lab[q], p);
        if (v > pb) {
            ps = pb;
            sec = best;
            pb = v;
            best = lab[q];
        } else if (v > ps) {
            ps = v;
            sec = lab[q];
        }
    }
    *second = sec;
    return best;
}

/* psi_ab and its cell gradient (src/opencl/v2m_seed_body.cl:179-247) */
static REAL FN(psi)(const FN(state)* s, int a, int b, const REAL* p) {
    REAL gv;
    if (FN(gray_psi)(s, a, b, p, &gv, NULL)) return gv;
    REAL u = p[0] / s->vx, v = p[1] / s->vy, w = p[2] / s->vz;
    int i0 = (int)FLOOR(u), j0 = (int)FLOOR(v), k0 = (int)FLOOR(w);
    REAL c[8], e[8];
    FN(cell)(s, a, i0, j0, k0, c);
    FN(cell)(s, b, i0, j0, k0, e);
    for (int m = 0; m < 8; ++m) c[m] -= e[m];
    return FN(blend)(c, u - i0, v - j0, w - k0);
}

static REAL FN(psi_grad)(const FN(state)* s, int a, int b, const REAL* p, REAL* g) {
    REAL gv;
    if (FN(gray_psi)(s, a, b, p, &gv, g)) return gv;
    REAL u = p[0] / s->vx, v = p[1] / s->vy, w = p[2] / s->vz;
    int i0 = (int)FLOOR(u), j0 = (int)FLOOR(v), k0 = (int)FLOOR(w);
    REAL fx = u - i0, fy = v - j0, fz = w - k0;
    REAL c[8], e[8];
    FN(cell)(s, a, i0, j0, k0, c);
    FN(cell)(s, b, i0, j0, k0, e);
    for (int m = 0; m < 8; ++m) c[m] -= e[m];
    REAL x00 = c[0] + fx * (c[1] - c[0]), x10 = c[2] + fx * (c[3] - c[2]);
    REAL x01 = c[4] + fx * (c[5] - c[4]), x11 = c[6] + fx * (c[7] - c[6]);
    REAL y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    REAL dx0 = (c[1] - c[0]) + fy * ((c[3] - c[2]) - (c[1] - c[0]));
    REAL dx1 = (c[5] - c[4]) + fy * ((c[7] - c[6]) - (c[5] - c[4]));
    g[0] = (dx0 + fz * (dx1 - dx0)) / s->vx;
    g[1] = ((x10 - x00) + fz * ((x11 - x01) - (x10 - x00))) / s->vy;
    g[2] = (y1 - y0) / s->vz;
    return y0 + fz * (y1 - y0);
}

/* bracketed root along u (src/opencl/v2m_seed_body.cl:255-320) */
static int FN(bisect)(const FN(state)* s, int a, int b, REAL* p, const REAL* u, REAL v0, REAL rad, REAL tg) {
    if (v0 == K(0.0)) return 1;
    REAL sg = v0 > K(0.0) ? K(-1.0) : K(1.0);
    REAL t0 = K(0.0), t1 = K(-1.0), f0 = v0, f1 = K(0.0);
    REAL t = (tg > K(0.0) && tg < rad) ? tg : K(0.25) * rad;
    for (int k = 0; k < 8; ++k) {
        REAL q[3] = { p[0] + sg * t * u[0], p[1] + sg * t * u[1], p[2] + sg * t * u[2] };
        REAL v = FN(psi)(s, a, b, q);
        if ((v > K(0.0)) != (v0 > K(0.0)) || v == K(0.0)) {
            t1 = t;
            f1 = v;
            break;
        }
        t0 = t;
        f0 = v;
        if (t >= rad) break;
        t = FMIN(K(2.0) * t, rad);
    }
    if (t1 < K(0.0)) return 0;
    int side = 0;
    for (int it = 0; it < 8 && f1 != K(0.0) && FABS(t1 - t0) > K(1e-4) * rad; ++it) {
        REAL tm = (f0 != f1) ? t1 - f1 * (t1 - t0) / (f1 - f0) : K(0.5) * (t0 + t1);
        REAL q[3] = { p[0] + sg * tm * u[0], p[1] + sg * tm * u[1], p[2] + sg * tm * u[2] };
        REAL v = FN(psi)(s, a, b, q);
        if ((v > K(0.0)) == (f1 > K(0.0))) {
            t1 = tm;
            f1 = v;
            if (side == -1) f0 *= K(0.5);
            side = -1;
        } else {
            t0 = t1;
            f0 = f1;
            t1 = tm;
            f1 = v;
            side = 1;
        }
    }
    for (int k = 0; k < 3; ++k) p[k] += sg * t1 * u[k];
    return 1;
}

static int FN(project1)(const FN(state)* s, int a, int b, REAL* p, REAL rad) {
    REAL g[3];
    REAL v = FN(psi_grad)(s, a, b, p, g);
    REAL gn = SQRT(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (gn < K(1e-9)) return 0;
    REAL u[3] = { g[0] / gn, g[1] / gn, g[2] / gn };
    return FN(bisect)(s, a, b, p, u, v, rad, K(1.5) * FABS(v) / gn);
}

/* src/opencl/v2m_seed_body.cl:342-420 */
static int FN(project2)(const FN(state)* s, int a, int b, int c, REAL* p, REAL rad) {
    REAL q[3] = { p[0], p[1], p[2] };
    if (s->gm < 0) { /* the pair of constraints with the most independent gradients, pivot first */
        REAL gab[3], gac[3], gbc[3];
        FN(psi_grad)(s, a, b, q, gab);
        FN(psi_grad)(s, a, c, q, gac);
        FN(psi_grad)(s, b, c, q, gbc);
        REAL xa[3] = { gab[1] * gac[2] - gab[2] * gac[1], gab[2] * gac[0] - gab[0] * gac[2], gab[0] * gac[1] - gab[1] * gac[0] };
        REAL xb[3] = { gab[1] * gbc[2] - gab[2] * gbc[1], gab[2] * gbc[0] - gab[0] * gbc[2], gab[0] * gbc[1] - gab[1] * gbc[0] };
        REAL xc[3] = { gac[1] * gbc[2] - gac[2] * gbc[1], gac[2] * gbc[0] - gac[0] * gbc[2], gac[0] * gbc[1] - gac[1] * gbc[0] };
        REAL na = xa[0] * xa[0] + xa[1] * xa[1] + xa[2] * xa[2], nb = xb[0] * xb[0] + xb[1] * xb[1] + xb[2] * xb[2],
             nc = xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2];
        if (nb > na && nb >= nc) {
            int t = a;
            a = b;
            b = t;
        } else if (nc > na && nc > nb) {
            int t = a;
            a = c;
            c = b;
            b = t;
        }
    }
    for (int it = 0; it < 3; ++it) {
        REAL g1[3], g2[3];
        if (!FN(project1)(s, a, b, q, rad)) return 0;
        FN(psi_grad)(s, a, b, q, g1);
        REAL v2 = FN(psi_grad)(s, a, c, q, g2);
        REAL a11 = g1[0] * g1[0] + g1[1] * g1[1] + g1[2] * g1[2];
        if (a11 < K(1e-18)) return 0;
        REAL pr = (g1[0] * g2[0] + g1[1] * g2[1] + g1[2] * g2[2]) / a11;
        REAL u[3] = { g2[0] - pr * g1[0], g2[1] - pr * g1[1], g2[2] - pr * g1[2] };
        REAL un = SQRT(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (un < K(1e-9)) return 0;
        u[0] /= un;
        u[1] /= un;
        u[2] /= un;
        if (!FN(bisect)(s, a, c, q, u, v2, rad, K(1.5) * FABS(v2) / un)) return 0;
    }
    if (!FN(project1)(s, a, b, q, rad)) return 0;
    REAL m2 = (q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]);
    if (m2 > rad * rad) return 0;
    p[0] = q[0];
    p[1] = q[1];
    p[2] = q[2];
    return 1;
}

/* src/opencl/v2m_particle_body.cl:188-291 */
static void FN(crossing)(const FN(state)* s, int a, int b, const REAL* p, const REAL* q, REAL* c) {
    REAL t0 = K(0.0), t1 = K(1.0);
    REAL v0 = FN(psi)(s, a, b, p), v1 = FN(psi)(s, a, b, q);
    for (int it = 0; it < 6; ++it) {
        REAL tm = K(0.5) * (t0 + t1);
        REAL x[3] = { p[0] + tm * (q[0] - p[0]), p[1] + tm * (q[1] - p[1]), p[2] + tm * (q[2] - p[2]) };
        REAL vm = FN(psi)(s, a, b, x);
        if (vm > K(0.0)) {
            t0 = tm;
            v0 = vm;
        } else {
            t1 = tm;
            v1 = vm;
        }
    }
    REAL t = (v0 - v1) != K(0.0) ? t0 + (t1 - t0) * v0 / (v0 - v1) : K(0.5) * (t0 + t1);
    for (int k = 0; k < 3; ++k) c[k] = p[k] + t * (q[k] - p[k]);
}

/* The constraint direction of every node at its position (the CUDA session's
   V2M_ARR_DIRS read): an INTERFACE node's unit normal of psi_(own, partner), a
   JUNCTION node's unit junction-line direction (the cross product of the two
   interface gradients the junction move of :926-945 below uses), zero for the
   other types and where the vector vanishes. */
static void FN(constraint_dirs)(const FN(state)* s, REAL* out) {
    for (int64_t i = 0; i < s->n; ++i) {
        const int ty = s->typ[i], a = s->lab[i], b = s->part[2 * i], c = s->part[2 * i + 1];
        REAL d[3] = { K(0.0), K(0.0), K(0.0) };
        if (ty == V2M_INTERFACE || ty == V2M_JUNCTION) {
            const REAL* p = s->P + 3 * i;
            REAL g1[3], u[3];
            FN(psi_grad)(s, a, b, p, g1);
            u[0] = g1[0];
            u[1] = g1[1];
            u[2] = g1[2];
            if (ty == V2M_JUNCTION) {
                REAL g2[3];
                FN(psi_grad)(s, a, c, p, g2);
                u[0] = g1[1] * g2[2] - g1[2] * g2[1];
                u[1] = g1[2] * g2[0] - g1[0] * g2[2];
                u[2] = g1[0] * g2[1] - g1[1] * g2[0];
            }
            const REAL un = SQRT(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
            if (un > K(0.0)) {
                d[0] = u[0] / un;
                d[1] = u[1] / un;
                d[2] = u[2] / un;
            }
        }
        out[3 * i] = d[0];
        out[3 * i + 1] = d[1];
        out[3 * i + 2] = d[2];
    }
}

static void FN(tangential)(const FN(state)* s, int a, int b, const REAL* p, REAL* v) {
    REAL g[3];
    FN(psi_grad)(s, a, b, p, g);
    REAL gn2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    if (gn2 < K(1e-12)) return;
    REAL vn = (v[0] * g[0] + v[1] * g[1] + v[2] * g[2]) / gn2;
    for (int k = 0; k < 3; ++k) v[k] -= vn * g[k];
}

static int FN(third)(const FN(state)* s, int a, int b, const REAL* q) {
    int nl[V2M_BL];
    int n = FN(labels_near)(s, q, nl), other = 0;
    for (int t = 0; t < n; ++t) other |= nl[t] != a && nl[t] != b;
    if (!other) return V2M_NOLAB;
    REAL pa = FN(phi_at)(s, a, q);
    int c = V2M_NOLAB;
    REAL pc = K(0.5) * pa;
    for (int t = 0; t < n; ++t) {
        if (nl[t] != a && nl[t] != b) {
            REAL w = FN(phi_at)(s, nl[t], q);
            if (w > pc) {
                pc = w;
                c = nl[t];
            }
        }
    }
    return c;
}

static int FN(valid_on)(const FN(state)* s, int a, int b, int c, const REAL* q) {
    int nl[V2M_BL];
    int n = FN(labels_near)(s, q, nl), other = 0;
    for (int t = 0; t < n; ++t) other |= nl[t] != a && nl[t] != b && nl[t] != c;
    if (!other) return 1;
    REAL mine = FMIN(FN(phi_at)(s, a, q), FN(phi_at)(s, b, q));
    if (c != V2M_NOLAB) mine = FMIN(mine, FN(phi_at)(s, c, q));
    for (int t = 0; t < n; ++t)
        if (nl[t] != a && nl[t] != b && nl[t] != c && FN(phi_at)(s, nl[t], q) > mine + K(0.02)) return 0;
    return 1;
}

/* ---- voxel trap mode (src/opencl/v2m_particle_body.cl:373-650) -------------------- */
static REAL FN(dda)(const FN(state)* s, int a, const REAL* p, const REAL* st, REAL* x, int* lb) {
    REAL vs[3] = { s->vx, s->vy, s->vz }, u[3], w[3];
    int id[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = p[k] / vs[k] + K(0.5);
        w[k] = st[k] / vs[k];
        id[k] = (int)FLOOR(u[k]);
    }
    int l = FN(label_at)(s, id[0], id[1], id[2]);
    if (l != a) {
        x[0] = p[0];
        x[1] = p[1];
        x[2] = p[2];
        *lb = l;
        return K(0.0);
    }
    REAL t = K(0.0);
    for (int it = 0; it < 64; ++it) {
        REAL ht[3];
        for (int k = 0; k < 3; ++k)
            ht[k] = w[k] != K(0.0) ? FABS(((REAL)id[k] + (w[k] > K(0.0) ? K(1.0) : K(0.0)) - u[k]) / w[k]) : K(1e30);
        REAL dt = FMIN(FMIN(ht[0], ht[1]), ht[2]);
        int ax = dt == ht[0] ? 0 : (dt == ht[1] ? 1 : 2);
        if (t + dt >= K(1.0)) return K(-1.0);
        t += dt;
        for (int k = 0; k < 3; ++k) u[k] += dt * w[k];
        u[ax] = (REAL)id[ax] + (w[ax] > K(0.0) ? K(1.0) : K(0.0));
        id[ax] += w[ax] > K(0.0) ? 1 : -1;
        l = FN(label_at)(s, id[0], id[1], id[2]);
        if (l != a) {
            for (int k = 0; k < 3; ++k) x[k] = (u[k] - K(0.5)) * vs[k];
            *lb = l;
            return t;
        }
    }
    return K(-1.0);
}

/* (q and out may alias: the reference passes the same array, and later
   candidates are measured from the updated point) */
static REAL FN(vox_nearest)(const FN(state)* s, int a, int b, int c, REAL* q, int R, REAL* out) {
    REAL vs[3] = { s->vx, s->vy, s->vz }, u[3];
    int ci[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = q[k] / vs[k] + K(0.5);
        ci[k] = (int)FLOOR(u[k]);
    }
    REAL best = K(-1.0);
    for (int vk = ci[2] - R; vk <= ci[2] + R; ++vk)
        for (int vj = ci[1] - R; vj <= ci[1] + R; ++vj)
            for (int vi = ci[0] - R; vi <= ci[0] + R; ++vi) {
                if (FN(label_at)(s, vi, vj, vk) != a) continue;
                int v[3] = { vi, vj, vk };
                for (int ax = 0; ax < 3; ++ax) {
                    int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
                    if (c == V2M_NOLAB) {
                        for (int sd = 0; sd < 2; ++sd) {
                            int nn[3] = { v[0], v[1], v[2] };
                            nn[ax] += sd ? 1 : -1;
                            if (FN(label_at)(s, nn[0], nn[1], nn[2]) != b) continue;
                            REAL y[3], d2 = K(0.0);
                            y[ax] = (REAL)(v[ax] + sd);
                            y[o1] = FMIN(FMAX(u[o1], (REAL)v[o1]), (REAL)(v[o1] + 1));
                            y[o2] = FMIN(FMAX(u[o2], (REAL)v[o2]), (REAL)(v[o2] + 1));
                            for (int k = 0; k < 3; ++k) {
                                y[k] = (y[k] - K(0.5)) * vs[k];
                                d2 += (y[k] - q[k]) * (y[k] - q[k]);
                            }
                            if (best < K(0.0) || d2 < best) {
                                best = d2;
                                out[0] = y[0];
                                out[1] = y[1];
                                out[2] = y[2];
                            }
                        }
                    } else {
                        for (int e = 0; e < 4; ++e) {
                            int e1 = e & 1, e2 = e >> 1, hb = 0, hc = 0;
                            for (int m = 0; m < 4; ++m) {
                                int nn[3] = { v[0], v[1], v[2] };
                                nn[o1] += e1 - 1 + (m & 1);
                                nn[o2] += e2 - 1 + (m >> 1);
                                int ln = FN(label_at)(s, nn[0], nn[1], nn[2]);
                                hb |= ln == b;
                                hc |= ln == c;
                            }
                            if (!hb || !hc) continue;
                            REAL y[3], d2 = K(0.0);
                            y[ax] = FMIN(FMAX(u[ax], (REAL)v[ax]), (REAL)(v[ax] + 1));
                            y[o1] = (REAL)(v[o1] + e1);
                            y[o2] = (REAL)(v[o2] + e2);
                            for (int k = 0; k < 3; ++k) {
                                y[k] = (y[k] - K(0.5)) * vs[k];
                                d2 += (y[k] - q[k]) * (y[k] - q[k]);
                            }
                            if (best < K(0.0) || d2 < best) {
                                best = d2;
                                out[0] = y[0];
                                out[1] = y[1];
                                out[2] = y[2];
                            }
                        }
                    }
                }
            }
    return best;
}

static int FN(vox_third)(const FN(state)* s, int a, int b, const REAL* p) {
    int i0 = (int)FLOOR(p[0] / s->vx), j0 = (int)FLOOR(p[1] / s->vy), k0 = (int)FLOOR(p[2] / s->vz);
    for (int m = 0; m < 8; ++m) {
        int l = FN(label_at)(s, i0 + (m & 1), j0 + ((m >> 1) & 1), k0 + (m >> 2));
        if (l != a && l != b) return l;
    }
    return V2M_NOLAB;
}

/* ---- size at a point (src/opencl/v2m_particle_body.cl:30-36; trilinear: extension) -- */
static REAL FN(h_at)(const FN(state)* s, const REAL* p) {
    if (s->hmode == 0) {
        int i = (int)FLOOR(p[0] / s->vx + K(0.5)), j = (int)FLOOR(p[1] / s->vy + K(0.5)), k = (int)FLOOR(p[2] / s->vz + K(0.5));
        i = i < 0 ? 0 : (i >= s->nx ? s->nx - 1 : i);
        j = j < 0 ? 0 : (j >= s->ny ? s->ny - 1 : j);
        k = k < 0 ? 0 : (k >= s->nz ? s->nz - 1 : k);
        return (REAL)s->hv[i + (size_t)s->nx * (j + (size_t)s->ny * k)];
    }
    REAL u = FMIN(FMAX(p[0] / s->vx, K(0.0)), (REAL)(s->nx - 1));
    REAL v = FMIN(FMAX(p[1] / s->vy, K(0.0)), (REAL)(s->ny - 1));
    REAL w = FMIN(FMAX(p[2] / s->vz, K(0.0)), (REAL)(s->nz - 1));
    int i0 = (int)FLOOR(u), j0 = (int)FLOOR(v), k0 = (int)FLOOR(w);
    if (i0 > s->nx - 2) i0 = s->nx > 1 ? s->nx - 2 : 0;
    if (j0 > s->ny - 2) j0 = s->ny > 1 ? s->ny - 2 : 0;
    if (k0 > s->nz - 2) k0 = s->nz > 1 ? s->nz - 2 : 0;
    int ii[2] = { i0, i0 + 1 < s->nx ? i0 + 1 : i0 }, jj[2] = { j0, j0 + 1 < s->ny ? j0 + 1 : j0 },
        kk[2] = { k0, k0 + 1 < s->nz ? k0 + 1 : k0 };
    REAL c[8];
    for (int m = 0; m < 8; ++m) c[m] = (REAL)s->hv[ii[m & 1] + (size_t)s->nx * (jj[(m >> 1) & 1] + (size_t)s->ny * kk[m >> 2])];
    return FN(blend)(c, u - i0, v - j0, w - k0);
}

/* ---- the move of node i (src/opencl/v2m_particle_body.cl:549-935) ---------------- */
static REAL FN(move_voxel)(FN(state)* s, REAL h, const REAL* st, int i) {
    REAL vmin = FMIN(FMIN(s->vx, s->vy), s->vz);
    REAL p[3] = { s->P[3 * i], s->P[3 * i + 1], s->P[3 * i + 2] }, q[3], x[3];
    int a = s->lab[i], ty = s->typ[i], b = s->part[2 * i], c = s->part[2 * i + 1];
    REAL sl = SQRT(st[0] * st[0] + st[1] * st[1] + st[2] * st[2]);
    int R = 1 + (int)CEIL(sl / vmin);
    for (int k = 0; k < 3; ++k) q[k] = p[k] + st[k];
    if (ty == V2M_INTERIOR) {
        int l;
        REAL t = FN(dda)(s, a, p, st, x, &l);
        if (t >= K(0.0)) {
            b = l;
            if (FN(vox_nearest)(s, a, b, V2M_NOLAB, q, R, q) < K(0.0)) {
                q[0] = x[0];
                q[1] = x[1];
                q[2] = x[2];
            }
            ty = V2M_INTERFACE;
        } else if (s->prm.snap > 0.0f) {
            REAL snap = (REAL)s->prm.snap;
            int Rs = 1 + (int)CEIL(snap * h / vmin);
            REAL best = K(-1.0), y[3];
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        int l2 = FN(label_at)(s, (int)FLOOR(q[0] / s->vx + K(0.5)) + dx * Rs,
                                              (int)FLOOR(q[1] / s->vy + K(0.5)) + dy * Rs,
                                              (int)FLOOR(q[2] / s->vz + K(0.5)) + dz * Rs);
                        if (l2 == a || l2 == b) continue;
                        REAL d2 = FN(vox_nearest)(s, a, l2, V2M_NOLAB, q, Rs, y);
                        if (d2 >= K(0.0) && d2 < snap * snap * h * h && (best < K(0.0) || d2 < best)) {
                            best = d2;
                            b = l2;
                            x[0] = y[0];
                            x[1] = y[1];
                            x[2] = y[2];
                        }
                    }
            if (best >= K(0.0)) {
                q[0] = x[0];
                q[1] = x[1];
                q[2] = x[2];
                ty = V2M_INTERFACE;
            }
        }
    } else if (ty == V2M_INTERFACE) {
        if (FN(vox_nearest)(s, a, b, V2M_NOLAB, q, R, q) < K(0.0)) return K(0.0);
    } else {
        if (FN(vox_nearest)(s, a, b, c, q, R, q) < K(0.0)) return K(0.0);
    }
    if (ty == V2M_INTERFACE) {
        int cc = FN(vox_third)(s, a, b, q);
        if (cc != V2M_NOLAB) {
            REAL r[3];
            REAL d2 = FN(vox_nearest)(s, a, b, cc, q, 1, r);
            if (d2 >= K(0.0) && d2 < K(0.0625) * h * h) {
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
                ty = V2M_JUNCTION;
                c = cc;
            }
        }
    }
    REAL mv = SQRT((q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]));
    s->P[3 * i] = q[0];
    s->P[3 * i + 1] = q[1];
    s->P[3 * i + 2] = q[2];
    s->typ[i] = (uint8_t)ty;
    s->part[2 * i] = (uint16_t)(ty == V2M_INTERIOR ? V2M_NOLAB : b);
    s->part[2 * i + 1] = (uint16_t)(ty >= V2M_JUNCTION ? c : V2M_NOLAB);
    s->hn[i] = FN(h_at)(s, q);
    return mv / h;
}

static REAL FN(move_step)(FN(state)* s, REAL h, REAL* st, int i) {
    const REAL maxstep = (REAL)s->prm.maxstep, snap = (REAL)s->prm.snap;
    REAL p[3] = { s->P[3 * i], s->P[3 * i + 1], s->P[3 * i + 2] }, q[3];
    const int a = s->lab[i], ty0 = s->typ[i];
    int ty = ty0;
    if (s->voxmode) return FN(move_voxel)(s, h, st, i);
    int b = s->part[2 * i];
    const int c = s->part[2 * i + 1];
    if (ty == V2M_INTERIOR) {
        for (int k = 0; k < 3; ++k) q[k] = p[k] + st[k];
        int sec;
        int l = FN(owner)(s, q, &sec);
        if (l != a) {
            b = l;
            REAL x[3], r[3];
            FN(crossing)(s, a, b, p, q, x);
            for (int k = 0; k < 3; ++k) r[k] = q[k] - x[k];
            FN(tangential)(s, a, b, x, r);
            for (int k = 0; k < 3; ++k) q[k] = x[k] + r[k];
            if (!FN(project1)(s, a, b, q, K(0.5) * h)) {
                q[0] = x[0];
                q[1] = x[1];
                q[2] = x[2];
            }
            ty = V2M_INTERFACE;
            s->part[2 * i] = (uint16_t)b;
        } else if (sec != V2M_NOLAB && snap > K(0.0)) {
            REAL gq[3];
            REAL v = FN(psi_grad)(s, a, sec, q, gq);
            REAL gn = SQRT(gq[0] * gq[0] + gq[1] * gq[1] + gq[2] * gq[2]);
            if (gn > K(1e-9) && v / gn < snap * h && FN(project1)(s, a, sec, q, K(1.2) * snap * h)) {
                ty = V2M_INTERFACE;
                b = sec;
                s->part[2 * i] = (uint16_t)sec;
            }
        }
    } else if (ty == V2M_INTERFACE) {
        FN(tangential)(s, a, b, p, st);
        for (int k = 0; k < 3; ++k) q[k] = p[k] + st[k];
        if (!FN(project1)(s, a, b, q, K(0.5) * h)) return K(0.0);
    } else {
        REAL g1[3], g2[3], td[3];
        FN(psi_grad)(s, a, b, p, g1);
        FN(psi_grad)(s, a, c, p, g2);
        td[0] = g1[1] * g2[2] - g1[2] * g2[1];
        td[1] = g1[2] * g2[0] - g1[0] * g2[2];
        td[2] = g1[0] * g2[1] - g1[1] * g2[0];
        REAL tl2 = td[0] * td[0] + td[1] * td[1] + td[2] * td[2];
        REAL sp = tl2 > K(1e-20) ? (st[0] * td[0] + st[1] * td[1] + st[2] * td[2]) / tl2 : K(0.0);
        for (int k = 0; k < 3; ++k) q[k] = p[k] + sp * td[k];
        if (!FN(project2)(s, a, b, c, q, K(0.5) * h)) return K(0.0);
    }
    if (ty == V2M_INTERFACE) {
        int cc = FN(third)(s, a, b, q);
        if (cc != V2M_NOLAB) {
            REAL r[3] = { q[0], q[1], q[2] };
            if (FN(project2)(s, a, b, cc, r, K(0.5) * h)) {
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
                ty = V2M_JUNCTION;
                s->part[2 * i + 1] = (uint16_t)cc;
            }
        }
    }
    {
        REAL lim = (maxstep + FMAX(snap, K(0.5))) * h;
        REAL m2 = (q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]);
        if (!(m2 <= lim * lim)) {
            if (ty0 == V2M_INTERIOR) s->part[2 * i] = V2M_NOLAB;
            return K(0.0);
        }
    }
    if (ty != V2M_INTERIOR &&
        !FN(valid_on)(s, a, s->part[2 * i], ty >= V2M_JUNCTION ? s->part[2 * i + 1] : V2M_NOLAB, q)) {
        if (ty == V2M_INTERFACE || ty0 == V2M_INTERIOR) {
            int cc = FN(third)(s, a, s->part[2 * i], q);
            REAL r[3] = { q[0], q[1], q[2] };
            if (cc != V2M_NOLAB && FN(project2)(s, a, s->part[2 * i], cc, r, K(0.5) * h) &&
                FN(valid_on)(s, a, s->part[2 * i], cc, r)) {
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
                ty = V2M_JUNCTION;
                s->part[2 * i + 1] = (uint16_t)cc;
            } else {
                if (ty0 == V2M_INTERIOR) s->part[2 * i] = V2M_NOLAB;
                return K(0.0);
            }
        } else {
            return K(0.0);
        }
    }
    REAL mv = SQRT((q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]));
    s->P[3 * i] = q[0];
    s->P[3 * i + 1] = q[1];
    s->P[3 * i + 2] = q[2];
    s->typ[i] = (uint8_t)ty;
    s->hn[i] = FN(h_at)(s, q);
    return mv / h;
}

static REAL FN(move)(FN(state)* s, int i) {
    REAL st[3];
    const REAL p0 = s->P[3 * i], p1 = s->P[3 * i + 1], p2 = s->P[3 * i + 2];
    const REAL pp[3] = { p0, p1, p2 };
    const REAL h = FN(h_at)(s, pp);
    const int ty0 = s->typ[i];
    const int fire = s->fire;
    const REAL maxstep = (REAL)s->prm.maxstep;
    if (fire) s->pw[i] = K(0.0);
    if (ty0 == V2M_CORNER) {
        if (fire) s->V[3 * i] = s->V[3 * i + 1] = s->V[3 * i + 2] = K(0.0);
        return K(0.0);
    }
    const REAL stiff = s->F[4 * i + 3] > K(1.0) ? s->F[4 * i + 3] : K(1.0);
    REAL ac[3];
    for (int k = 0; k < 3; ++k) ac[k] = s->F[4 * i + k] / stiff;
    if (fire) {
        REAL v[3] = { s->V[3 * i], s->V[3 * i + 1], s->V[3 * i + 2] };
        REAL pv = ac[0] * v[0] + ac[1] * v[1] + ac[2] * v[2];
        s->pw[i] = pv;
        if (pv < K(0.0)) {
            v[0] = v[1] = v[2] = K(0.0);
        } else {
            REAL vn = SQRT(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            REAL an = SQRT(ac[0] * ac[0] + ac[1] * ac[1] + ac[2] * ac[2]);
            if (an > K(0.0))
                for (int k = 0; k < 3; ++k) v[k] = (K(1.0) - s->falpha) * v[k] + s->falpha * vn * ac[k] / an;
        }
        for (int k = 0; k < 3; ++k) {
            v[k] += s->fdt * ac[k];
            st[k] = s->fdt * v[k];
        }
    } else {
        for (int k = 0; k < 3; ++k) st[k] = (REAL)s->prm.dt * ac[k];
    }
    REAL sl = SQRT(st[0] * st[0] + st[1] * st[1] + st[2] * st[2]);
    if (sl < K(5e-4) * h) {
        if (fire) s->V[3 * i] = s->V[3 * i + 1] = s->V[3 * i + 2] = K(0.0);
        return K(0.0);
    }
    if (sl > maxstep * h)
        for (int k = 0; k < 3; ++k) st[k] *= maxstep * h / sl;
    REAL m = FN(move_step)(s, h, st, i);
    if (fire) {
        if (m > K(0.0) && s->typ[i] == ty0) {
            s->V[3 * i] = (s->P[3 * i] - p0) / s->fdt;
            s->V[3 * i + 1] = (s->P[3 * i + 1] - p1) / s->fdt;
            s->V[3 * i + 2] = (s->P[3 * i + 2] - p2) / s->fdt;
        } else {
            s->V[3 * i] = s->V[3 * i + 1] = s->V[3 * i + 2] = K(0.0);
        }
    }
    return m;
}

/* ---- hash and lists (src/opencl/v2m_particle_body.cl:38-151) ---------------------- */
static int FN(level_of)(const FN(state)* s, REAL R) {
    int L = 0;
    while (L + 1 < s->nlev && s->b0 * (REAL)(1 << L) < R) ++L;
    return L;
}

static int FN(bin_coord)(const FN(state)* s, int L, REAL x, REAL o, int ax) {
    int c = (int)FLOOR((x - o) / (s->b0 * (REAL)(1 << L)));
    int n = s->dim[L][ax];
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

typedef struct {
    REAL d;
    int id;
} FN(cand);

static int FN(cand_cmp)(const void* x, const void* y) {
    const FN(cand)* a = (const FN(cand)*)x;
    const FN(cand)* b = (const FN(cand)*)y;
    if (a->d < b->d) return -1;
    if (a->d > b->d) return 1;
    return (a->id > b->id) - (a->id < b->id);
}

/* All candidates within reach, then the K smallest by (distance, id). */
static void FN(neighbors)(FN(state)* s, int i, FN(cand)** buf, int* cap) {
    const REAL px = s->P[3 * i], py = s->P[3 * i + 1], pz = s->P[3 * i + 2];
    const REAL hi = s->hn[i];
    const REAL ts = (REAL)s->prm.t + (REAL)s->prm.skin;
    const REAL Ri = ts * hi;
    const int interior = s->typ[i] == V2M_INTERIOR, li = s->lab[i];
    const int Li = FN(level_of)(s, Ri);
    int m = 0;
    for (int L = Li - 1; L <= Li + 1; ++L) {
        if (L < 0 || L >= s->nlev) continue;
        REAL bL = s->b0 * (REAL)(1 << L), r = K(0.5) * (Ri + bL);
        int x0 = FN(bin_coord)(s, L, px - r, s->ox, 0), x1 = FN(bin_coord)(s, L, px + r, s->ox, 0);
        int y0 = FN(bin_coord)(s, L, py - r, s->oy, 1), y1 = FN(bin_coord)(s, L, py + r, s->oy, 1);
        int z0 = FN(bin_coord)(s, L, pz - r, s->oz, 2), z1 = FN(bin_coord)(s, L, pz + r, s->oz, 2);
        for (int cz = z0; cz <= z1; ++cz)
            for (int cy = y0; cy <= y1; ++cy)
                for (int cx = x0; cx <= x1; ++cx) {
                    int key = s->off[L] + cx + s->dim[L][0] * (cy + s->dim[L][1] * cz);
                    for (int q = s->cstart[key]; q < s->cstart[key + 1]; ++q) {
                        int j = s->sorted[q];
                        if (j == i) continue;
                        REAL ex = s->Ps[4 * q] - px, ey = s->Ps[4 * q + 1] - py, ez = s->Ps[4 * q + 2] - pz;
                        REAL d2 = ex * ex + ey * ey + ez * ez;
                        REAL rj = ts * K(0.5) * (hi + s->Ps[4 * q + 3]);
                        if (d2 >= rj * rj) continue;
                        if (interior && s->typ[j] == V2M_INTERIOR && s->lab[j] != li) continue;
                        if (m == *cap) {
                            *cap = *cap ? 2 * *cap : 256;
                            *buf = (FN(cand)*)realloc(*buf, sizeof(FN(cand)) * (size_t)*cap);
                        }
                        (*buf)[m].d = SQRT(d2);
                        (*buf)[m].id = j;
                        ++m;
                    }
                }
    }
    qsort(*buf, (size_t)m, sizeof(FN(cand)), FN(cand_cmp));
    int n = m < V2M_K ? m : V2M_K;
    s->nnb[i] = n;
    for (int k = 0; k < n; ++k) s->nbr[(size_t)i * V2M_K + k] = (*buf)[k].id;
}

/* ---- the driver (src/v2m_particles.cpp:728-946) -------------------------------------- */
static void FN(free)(FN(state)* s) {
    if (!s) return;
    free(s->P); free(s->P0); free(s->hn); free(s->F); free(s->V); free(s->pw); free(s->mv); free(s->Ps);
    free(s->lab); free(s->typ); free(s->part); free(s->key); free(s->cstart); free(s->sorted); free(s->nbr);
    free(s->nnb);
    free(s);
}

static FN(state)* FN(create)(const v2m_grid_view* g, const v2m_relax_params* p, const v2m_nodes_view* nd) {
    FN(state)* s = (FN(state)*)calloc(1, sizeof(FN(state)));
    if (!s) return NULL;
    s->nx = g->nx; s->ny = g->ny; s->nz = g->nz; s->nbx = g->nbx; s->nby = g->nby; s->nbz = g->nbz;
    s->vx = (REAL)g->vs[0]; s->vy = (REAL)g->vs[1]; s->vz = (REAL)g->vs[2];
    s->L = g->L; s->bl_cnt = g->bl_cnt; s->bl_lab = g->bl_lab; s->bl_slot = g->bl_slot; s->phi = g->phi;
    s->hv = g->h; s->gI = g->gI; s->gTW = g->gTW; s->gm = g->gm; s->hmin = g->hmin; s->hmax = g->hmax;
    s->ntw = g->gm < 0 ? g->ngTW : (g->gm > 0 ? 2 * (int64_t)g->gm : 0);
    s->prm = *p;
    s->fire = p->fire && !p->voxel_trap;
    s->voxmode = p->voxel_trap != 0;
    s->hmode = p->h_mode;
    s->rebuild_div = p->rebuild_div > 0 ? p->rebuild_div : (getenv("V2M_REBUILD_DIV") ? atoi(getenv("V2M_REBUILD_DIV")) : 300);
    if (s->rebuild_div < 1) s->rebuild_div = 1;
    /* hash geometry (src/v2m_particles.cpp:737-761) */
    const REAL ts = (REAL)p->t + (REAL)p->skin;
    s->b0 = ts * (REAL)g->hmin;
    s->ox = K(-0.5) * s->vx;
    s->oy = K(-0.5) * s->vy;
    s->oz = K(-0.5) * s->vz;
    REAL ext[3] = { g->nx * s->vx, g->ny * s->vy, g->nz * s->vz };
    s->nlev = 1;
    while (s->nlev < V2M_MAXLEV && s->b0 * (REAL)(1 << (s->nlev - 1)) < ts * (REAL)g->hmax) ++s->nlev;
    int nk = 0;
    for (int L = 0; L < s->nlev; ++L) {
        s->off[L] = nk;
        REAL bL = s->b0 * (REAL)(1 << L);
        for (int a = 0; a < 3; ++a) {
            int d = (int)CEIL(ext[a] / bL);
            s->dim[L][a] = d < 1 ? 1 : d;
        }
        nk += s->dim[L][0] * s->dim[L][1] * s->dim[L][2];
    }
    s->nkeys = nk;
    int n = (int)nd->n;
    s->n = n;
    size_t nn = (size_t)(n > 0 ? n : 1);
    s->P = (REAL*)malloc(sizeof(REAL) * 3 * nn);
    s->P0 = (REAL*)malloc(sizeof(REAL) * 3 * nn);
    s->hn = (REAL*)malloc(sizeof(REAL) * nn);
    s->F = (REAL*)calloc(4 * nn, sizeof(REAL));
    s->V = (REAL*)calloc(3 * nn, sizeof(REAL));
    s->pw = (REAL*)calloc(nn, sizeof(REAL));
    s->mv = (REAL*)calloc(nn, sizeof(REAL));
    s->Ps = (REAL*)calloc(4 * nn, sizeof(REAL));
    s->lab = (uint16_t*)malloc(2 * nn);
    s->typ = (uint8_t*)malloc(nn);
    s->part = (uint16_t*)malloc(4 * nn);
    s->key = (int*)calloc(nn, sizeof(int));
    s->cstart = (int*)calloc((size_t)nk + 1, sizeof(int));
    s->sorted = (int*)calloc(nn, sizeof(int));
    s->nbr = (int*)calloc(nn * V2M_K, sizeof(int));
    s->nnb = (int*)calloc(nn, sizeof(int));
    for (int i = 0; i < 3 * n; ++i) s->P[i] = (REAL)nd->P[i];
    if (n > 0) {
        memcpy(s->lab, nd->lab, 2 * (size_t)n);
        memcpy(s->typ, nd->typ, (size_t)n);
        memcpy(s->part, nd->part, 4 * (size_t)n);
    }
    memcpy(s->P0, s->P, sizeof(REAL) * 3 * (size_t)n);
    for (int i = 0; i < n; ++i) s->hn[i] = FN(h_at)(s, s->P + 3 * i);
    s->fdt0 = SQRT((REAL)p->dt);
    s->fdt = s->fdt0;
    s->fdtmax = (REAL)p->fire_dtmax * s->fdt0;
    s->falpha = K(0.1);
    return s;
}

static void FN(rebuild)(FN(state)* s) {
    const int n = s->n;
    const REAL ts = (REAL)s->prm.t + (REAL)s->prm.skin;
    for (int i = 0; i < n; ++i) {
        REAL h = FN(h_at)(s, s->P + 3 * i);
        int L = FN(level_of)(s, ts * h);
        int cx = FN(bin_coord)(s, L, s->P[3 * i], s->ox, 0), cy = FN(bin_coord)(s, L, s->P[3 * i + 1], s->oy, 1),
            cz = FN(bin_coord)(s, L, s->P[3 * i + 2], s->oz, 2);
        s->key[i] = s->off[L] + cx + s->dim[L][0] * (cy + s->dim[L][1] * cz);
    }
    memset(s->cstart, 0, sizeof(int) * ((size_t)s->nkeys + 1));
    for (int i = 0; i < n; ++i) ++s->cstart[s->key[i] + 1];
    for (int k = 0; k < s->nkeys; ++k) s->cstart[k + 1] += s->cstart[k];
    int* cur = (int*)malloc(sizeof(int) * ((size_t)s->nkeys + 1));
    memcpy(cur, s->cstart, sizeof(int) * ((size_t)s->nkeys + 1));
    for (int i = 0; i < n; ++i) s->sorted[cur[s->key[i]]++] = i;
    free(cur);
    for (int q = 0; q < n; ++q) {
        int j = s->sorted[q];
        s->Ps[4 * q] = s->P[3 * j];
        s->Ps[4 * q + 1] = s->P[3 * j + 1];
        s->Ps[4 * q + 2] = s->P[3 * j + 2];
        s->Ps[4 * q + 3] = s->hn[j];
    }
    FN(cand)* buf = NULL;
    int cap = 0;
    for (int i = 0; i < n; ++i) FN(neighbors)(s, i, &buf, &cap);
    free(buf);
    memcpy(s->P0, s->P, sizeof(REAL) * 3 * (size_t)n);
    ++s->rebuilds;
}

/* src/opencl/v2m_particle_body.cl:161-184 */
static void FN(force)(FN(state)* s) {
    const REAL fscale = (REAL)s->prm.fscale, fsurf = (REAL)s->prm.fsurf;
    for (int i = 0; i < s->n; ++i) {
        const REAL px = s->P[3 * i], py = s->P[3 * i + 1], pz = s->P[3 * i + 2], hi = s->hn[i];
        REAL f4[4] = { K(0.0), K(0.0), K(0.0), K(0.0) };
        for (int k = 0; k < s->nnb[i]; ++k) {
            int j = s->nbr[(size_t)i * V2M_K + k];
            REAL ex = px - s->P[3 * j], ey = py - s->P[3 * j + 1], ez = pz - s->P[3 * j + 2];
            REAL l = SQRT(ex * ex + ey * ey + ez * ez);
            REAL l0 = ((s->typ[i] != V2M_INTERIOR && s->typ[j] != V2M_INTERIOR) ? fsurf : fscale) * K(0.5) * (hi + s->hn[j]);
            if (l >= l0 || l <= K(0.0)) continue;
            REAL f = (l0 - l) / l;
            f4[0] += f * ex;
            f4[1] += f * ey;
            f4[2] += f * ez;
            f4[3] += K(1.0);
        }
        for (int k = 0; k < 4; ++k) s->F[4 * i + k] = f4[k];
    }
}

static void FN(move_all)(FN(state)* s) {
    REAL mmax = K(0.0);
    for (int i = 0; i < s->n; ++i) {
        s->mv[i] = FN(move)(s, i);
        if (s->mv[i] > mmax) mmax = s->mv[i];
    }
    s->mmax = mmax;
}

/* the rest of one iteration; returns 1 on convergence */
static int FN(tail)(FN(state)* s) {
    const int n = s->n, it = s->it;
    FN(move_all)(s);
    if (s->fire) {
        double pt = 0.0;
        for (int i = 0; i < n; ++i) pt += (double)s->pw[i];
        s->power = pt;
        if (pt >= 0.0) { /* FireCtl::update, src/v2m_particles.h:58-73 */
            if (++s->npos > 5) {
                s->fdt = FMIN(s->fdt * K(1.1), s->fdtmax);
                s->falpha *= K(0.99);
            }
        } else {
            s->npos = 0;
            s->fdt = FMAX(s->fdt * K(0.5), K(0.05) * s->fdt0);
            s->falpha = K(0.1);
            ++s->resets;
            memset(s->V, 0, sizeof(REAL) * 3 * (size_t)n);
        }
    }
    memset(s->hist, 0, sizeof(s->hist));
    for (int i = 0; i < n; ++i) {
        double m = (double)s->mv[i];
        int b = 0;
        if (m > 0.0) {
            b = 20 + (int)floor((double)(float)log2(m));
            b = b < 0 ? 0 : (b > 31 ? 31 : b);
        }
        ++s->hist[b];
    }
    int acc = 0, b99 = 31;
    for (int b = 0; b < 32; ++b) {
        acc += s->hist[b];
        if (acc >= 0.99 * n) {
            b99 = b;
            break;
        }
    }
    s->p99 = (REAL)ldexpf(1.0f, b99 - 20 + 1);
    s->it = it + 1;
    if (s->p99 < (REAL)s->prm.dptol && (!s->fire || s->fdt >= K(0.25) * s->fdt0)) {
        s->stopped = 1;
        return 1;
    }
    int nhalf = 0, nref = 0;
    const REAL skin = (REAL)s->prm.skin;
    const int policy = s->prm.rebuild_policy;   /* extensions: 1 max displacement, 2 fixed lists */
    REAL maxd = K(0.0);
    FN(cand)* buf = NULL;
    int cap = 0;
    for (int i = 0; i < n; ++i) {
        REAL ex = s->P[3 * i] - s->P0[3 * i], ey = s->P[3 * i + 1] - s->P0[3 * i + 1], ez = s->P[3 * i + 2] - s->P0[3 * i + 2];
        REAL h = FN(h_at)(s, s->P + 3 * i);
        REAL m2 = ex * ex + ey * ey + ez * ez, s2 = skin * skin * h * h;
        if (policy == 1) {
            const REAL d = SQRT(m2) / h;
            maxd = d > maxd ? d : maxd;
        }
        if (m2 > s2 && policy != 2) {
            FN(neighbors)(s, i, &buf, &cap);
            s->P0[3 * i] = s->P[3 * i];
            s->P0[3 * i + 1] = s->P[3 * i + 1];
            s->P0[3 * i + 2] = s->P[3 * i + 2];
            ++nref;
        } else {
            nhalf += m2 > K(0.25) * s2;
        }
    }
    free(buf);
    s->nhalf = nhalf;
    s->nrefresh = nref;
    if (policy == 1) {
        if (maxd > K(0.1)) FN(rebuild)(s);
        return 0;
    }
    if (policy == 2) return 0;   /* the first build's lists for the whole run */
    int endgame = it >= s->prm.max_iters * 4 / 5 || s->p99 < K(4.0) * (REAL)s->prm.dptol;
    int div = endgame ? (s->rebuild_div > 1000 ? s->rebuild_div : 1000) : s->rebuild_div;
    if (nhalf > n / div) FN(rebuild)(s);
    return 0;
}
