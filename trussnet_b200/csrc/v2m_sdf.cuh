// v2m_sdf.cuh -- the analytic shape fields (gm < 0) on the device.
//
// Shape input carries, per label, a compiled postfix program of signed distance
// terms (the layout of src/opencl/v2m_sdf_body.cl:9-21, written by the
// reference's shape compiler, src/v2m_sdfshape.cpp): s_l > 0 inside label l,
// world units. The relaxation's point queries then read phi_l =
// clamp(0.5 + s_l / w) and psi_ab = (s_a - s_b) / w instead of the sampled
// fields (src/opencl/v2m_seed_body.cl:29-37, 162-165, 182-184, 214-221).
//
// Program layout (floats): [0] N labels, [1] w, [2..4] origin (world = grid mm +
// origin), [5 .. 5+N) code offsets, [5+N] crease blend radius, [6+N] gap-closing
// radius, [7+N] cull margin, [8+N] brick table offset (0: none; at T: nbx nby nbz
// voxel, then per brick the offset of its N code offsets). A code is a sequence
// of opcodes with operands, ended by END.
//
// Every float expression keeps the reference's operand order (the kernels are
// compiled without FMA contraction), so the values are the reference's bit for
// bit. Every read of the program is bounds-checked against its length: a
// malformed program ends its evaluation (as the reference's own "malformed"
// exit) instead of reading past the buffer.
#pragma once

#include "v2m_types.cuh"

namespace v2m {
// (internal linkage: the header is compiled into more than one source)
namespace {

enum SdfOp : int {
    kSdfEnd = 0,
    kSdfPrim = 1,     // type, parameters
    kSdfMax = 2,      // union
    kSdfMin = 3,      // intersection
    kSdfNeg = 4,      // complement
    kSdfConst = 5,    // value
    kSdfBbox = 6,     // lo[3] hi[3] len f
    kSdfMconst = 7,   // f x the cull margin
    kSdfAdd = 8,
    kSdfScale = 9,
    kSdfCmax = 10,    // union inside one object (no gap closing)
    kSdfCmin = 11,    // intersection inside one object
};

enum SdfPrim : int {
    kPrimSphere = 1,
    kPrimBox = 2,
    kPrimCyl = 3,
    kPrimPlane = 4,
    kPrimSlab = 5,
    kPrimTorus = 6,
    kPrimEllipsoid = 7,
    kPrimCone = 8,
    kPrimInfCyl = 9,
};

constexpr int kSdfStack = 12;   // the deepest stack a program may use (the shape compiler checks it)

// value and gradient of a stack entry
struct SdfV {
    float v, x, y, z;
};

__device__ __forceinline__ SdfV sdf_zero() {
    SdfV r;
    r.v = r.x = r.y = r.z = 0.0f;
    return r;
}

__device__ __forceinline__ int sdf_nparam(int type) {
    switch (type) {
    case kPrimSphere:
        return 4;
    case kPrimBox:
    case kPrimPlane:
        return 6;
    case kPrimCyl:
    case kPrimInfCyl:
        return 7;
    case kPrimSlab:
    case kPrimTorus:
    case kPrimCone:
        return 8;
    case kPrimEllipsoid:
        return 15;
    default:
        return 0;
    }
}

// One primitive's signed distance at world point (x, y, z), > 0 inside
// (src/opencl/v2m_sdf_body.cl:75-167: the same formulas and operand order).
__device__ __forceinline__ float sdf_prim(int type, const float* __restrict__ q, float x, float y, float z) {
    switch (type) {
    case kPrimSphere: {
        const float dx = x - q[0], dy = y - q[1], dz = z - q[2];
        return q[3] - sqrtf(dx * dx + dy * dy + dz * dz);
    }
    case kPrimBox: {
        const float cx = 0.5f * (q[0] + q[3]), cy = 0.5f * (q[1] + q[4]), cz = 0.5f * (q[2] + q[5]);
        const float ux = fabsf(x - cx) - 0.5f * fabsf(q[3] - q[0]);
        const float uy = fabsf(y - cy) - 0.5f * fabsf(q[4] - q[1]);
        const float uz = fabsf(z - cz) - 0.5f * fabsf(q[5] - q[2]);
        const float ox = fmaxf(ux, 0.0f), oy = fmaxf(uy, 0.0f), oz = fmaxf(uz, 0.0f);
        const float out = sqrtf(ox * ox + oy * oy + oz * oz);
        const float in = fminf(fmaxf(ux, fmaxf(uy, uz)), 0.0f);
        return -(out + in);
    }
    case kPrimPlane:
        return -((x - q[0]) * q[3] + (y - q[1]) * q[4] + (z - q[2]) * q[5]);
    case kPrimSlab: {
        const float t = (x - q[0]) * q[3] + (y - q[1]) * q[4] + (z - q[2]) * q[5];
        return fminf(t - q[6], q[7] - t);
    }
    case kPrimInfCyl: {
        const float dx = x - q[0], dy = y - q[1], dz = z - q[2];
        const float t = dx * q[3] + dy * q[4] + dz * q[5];
        const float rx = dx - t * q[3], ry = dy - t * q[4], rz = dz - t * q[5];
        return q[6] - sqrtf(rx * rx + ry * ry + rz * rz);
    }
    case kPrimTorus: {
        const float dx = x - q[0], dy = y - q[1], dz = z - q[2];
        const float h = dx * q[3] + dy * q[4] + dz * q[5];
        const float rx = dx - h * q[3], ry = dy - h * q[4], rz = dz - h * q[5];
        const float a = sqrtf(rx * rx + ry * ry + rz * rz) - q[6];
        return q[7] - sqrtf(a * a + h * h);
    }
    case kPrimCyl: {   // capped cylinder, exact
        const float bx = q[3] - q[0], by = q[4] - q[1], bz = q[5] - q[2];
        const float px = x - q[0], py = y - q[1], pz = z - q[2];
        const float baba = bx * bx + by * by + bz * bz, paba = px * bx + py * by + pz * bz;
        const float ex = px * baba - bx * paba, ey = py * baba - by * paba, ez = pz * baba - bz * paba;
        const float u = sqrtf(ex * ex + ey * ey + ez * ez) - q[6] * baba;
        const float v = fabsf(paba - baba * 0.5f) - baba * 0.5f;
        const float u2 = u * u, v2 = v * v * baba;
        const float dd = fmaxf(u, v) < 0.0f ? -fminf(u2, v2) : ((u > 0.0f ? u2 : 0.0f) + (v > 0.0f ? v2 : 0.0f));
        return -(dd < 0.0f ? -1.0f : 1.0f) * sqrtf(fabsf(dd)) / baba;
    }
    case kPrimCone: {   // capped frustum a (radius ra) .. b (radius rb), exact
        const float bx = q[3] - q[0], by = q[4] - q[1], bz = q[5] - q[2];
        const float px = x - q[0], py = y - q[1], pz = z - q[2];
        const float ra = q[6], rb = q[7];
        const float rba = rb - ra, baba = bx * bx + by * by + bz * bz;
        const float papa = px * px + py * py + pz * pz, paba = (px * bx + py * by + pz * bz) / baba;
        const float xr = sqrtf(fmaxf(papa - paba * paba * baba, 0.0f));
        const float cax = fmaxf(0.0f, xr - ((paba < 0.5f) ? ra : rb)), cay = fabsf(paba - 0.5f) - 0.5f;
        const float k = rba * rba + baba;
        const float f = fminf(fmaxf((rba * (xr - ra) + paba * baba) / k, 0.0f), 1.0f);
        const float cbx = xr - ra - f * rba, cby = paba - f;
        const float sg = (cbx < 0.0f && cay < 0.0f) ? -1.0f : 1.0f;
        const float d2 = fminf(cax * cax + cay * cay * baba, cbx * cbx + cby * cby * baba);
        return -sg * sqrtf(d2);
    }
    case kPrimEllipsoid: {   // a bound, exact on the surface: k0 (k0 - 1) / k1
        const float dx = x - q[0], dy = y - q[1], dz = z - q[2];
        const float lx = q[6] * dx + q[7] * dy + q[8] * dz;
        const float ly = q[9] * dx + q[10] * dy + q[11] * dz;
        const float lz = q[12] * dx + q[13] * dy + q[14] * dz;
        const float ax = lx / q[3], ay = ly / q[4], az = lz / q[5];
        const float bx = ax / q[3], by = ay / q[4], bz = az / q[5];
        const float k0 = sqrtf(ax * ax + ay * ay + az * az), k1 = sqrtf(bx * bx + by * by + bz * bz);
        if (k1 < 1e-20f) {
            return fminf(q[3], fminf(q[4], q[5]));
        }
        return -k0 * (k0 - 1.0f) / k1;
    }
    default:
        return -1e30f;
    }
}

// min (sgn 1) or max (sgn -1) of a and b with the crease blend (radius k) and
// the gap closing (radius kgap) of src/opencl/v2m_sdf_body.cl:174-259. Without
// the gradients, *near is set where the result would need them (a possible
// sliver, or a blend whose fade depends on the gradients' angle).
__device__ __forceinline__ SdfV sdf_minmax(SdfV a, SdfV b, float sgn, float k, float kgap, int grad, int* near) {
    const float va = sgn * a.v, vb = sgn * b.v;
    const bool sliver = kgap > 0.0f && va > -kgap && vb > -kgap && va + vb < kgap;
    if (sliver && !grad) {
        *near = 1;
    }
    float pen = 0.0f, dpen = 0.0f;
    if (sliver && grad) {
        // facing surfaces closer than kgap: the penalty kgap wg u^2 closes the gap
        const float ga = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z), gb = sqrtf(b.x * b.x + b.y * b.y + b.z * b.z);
        if (ga > 0.0f && gb > 0.0f) {
            const float c = (a.x * b.x + a.y * b.y + a.z * b.z) / (ga * gb);
            const float wg = fminf(1.0f, fmaxf(0.0f, (-c - 0.7f) / 0.25f));
            const float u = fmaxf(0.0f, 1.0f - (va + vb) / kgap);
            pen = kgap * wg * u * u;
            dpen = 2.0f * wg * u;
        }
    }
    SdfV r = a;
    if (k > 0.0f && fabsf(va - vb) < k) {
        // no crease to round where the two surfaces lie on each other: the
        // blend fades out as the gradients align
        if (!grad) {
            *near = 1;
        } else {
            const float ga = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z), gb = sqrtf(b.x * b.x + b.y * b.y + b.z * b.z);
            const float c = ga > 0.0f && gb > 0.0f ? (a.x * b.x + a.y * b.y + a.z * b.z) / (ga * gb) : 0.0f;
            k *= fminf(1.0f, fmaxf(0.0f, (0.995f - c) / 0.095f));
        }
    }
    if (k > 0.0f && fabsf(va - vb) < k) {
        // quadratic smooth min within k of the crease
        const float h = 0.5f + 0.5f * (vb - va) / k;
        r.v = sgn * (vb * (1.0f - h) + va * h - k * h * (1.0f - h));
        r.x = h * a.x + (1.0f - h) * b.x;
        r.y = h * a.y + (1.0f - h) * b.y;
        r.z = h * a.z + (1.0f - h) * b.z;
    } else if (vb < va) {
        r = b;
    }
    r.v -= sgn * pen;
    if (dpen > 0.0f) {
        r.x += dpen * (a.x + b.x);
        r.y += dpen * (a.y + b.y);
        r.z += dpen * (a.z + b.z);
    }
    return r;
}

// The program's float at index k, or END (0) outside it.
__device__ __forceinline__ float sdf_at(const DGrid& g, int64_t k) {
    return (k >= 0 && k < g.ntw) ? __ldg(g.gTW + k) : 0.0f;
}

__device__ __forceinline__ bool sdf_is_minmax(int op) {
    return op == kSdfMax || op == kSdfMin || op == kSdfCmax || op == kSdfCmin;
}

// s_l at grid-mm point p and, with wantg, its gradient
// (src/opencl/v2m_sdf_body.cl:262-478). The stack's top four entries live in
// registers (t0 the top), deeper ones in `deep`. A first pass runs without
// gradients unless asked; a second runs with them only where a min / max met a
// possible gap or blend fade.
__device__ __noinline__ SdfV sdf_evalv(const DGrid& g, int l, float px, float py, float pz, int wantg) {
    const int N = (int)sdf_at(g, 0);
    SdfV none = sdf_zero();
    none.v = -1e30f;
    if (l < 0 || l >= N) {
        return none;
    }
    const float x = px + sdf_at(g, 2), y = py + sdf_at(g, 3), z = pz + sdf_at(g, 4);
    int start = (int)sdf_at(g, 5 + l);
    {
        const int T = (int)sdf_at(g, 8 + N);
        if (T > 0) {
            // the point's brick's own program (only the objects near it)
            const int nbx = (int)sdf_at(g, T), nby = (int)sdf_at(g, T + 1), nbz = (int)sdf_at(g, T + 2);
            const float vx = sdf_at(g, T + 3);
            int bi = (int)floorf(px / vx + 0.5f) >> 3, bj = (int)floorf(py / vx + 0.5f) >> 3,
                bk = (int)floorf(pz / vx + 0.5f) >> 3;
            bi = bi < 0 ? 0 : (bi >= nbx ? nbx - 1 : bi);
            bj = bj < 0 ? 0 : (bj >= nby ? nby - 1 : bj);
            bk = bk < 0 ? 0 : (bk >= nbz ? nbz - 1 : bk);
            const int64_t e = (int64_t)T + 4 + bi + (int64_t)nbx * (bj + (int64_t)nby * bk);
            start = (int)sdf_at(g, (int64_t)(int)sdf_at(g, e) + l);
        }
    }
    const float kblend = sdf_at(g, 5 + N), kgap = sdf_at(g, 6 + N), margin = sdf_at(g, 7 + N);
    SdfV t0 = sdf_zero(), t1 = t0, t2 = t0, t3 = t0;
    SdfV deep[kSdfStack - 4];
    int sp = 0;
    int grad = wantg != 0;
    for (int pass = 0; pass < 2; ++pass) {
        sp = 0;
        int pc = start, near = 0;
        for (int guard = 0; guard < 100000; ++guard) {
            const int op = (int)sdf_at(g, pc);
            if (op == kSdfEnd) {
                break;
            }
            if (sdf_is_minmax(op)) {   // t1 op t0 -> t0
                if (sp > 1) {
                    t0 = sdf_minmax(t1, t0, op == kSdfMax || op == kSdfCmax ? -1.0f : 1.0f, kblend,
                                    op >= kSdfCmax ? 0.0f : kgap, grad, &near);
                    t1 = t2;
                    t2 = t3;
                    if (sp > 4) {
                        t3 = deep[sp - 5];
                    }
                    --sp;
                }
                pc += 1;
                continue;
            }
            if (op == kSdfNeg) {
                t0.v = -t0.v;
                t0.x = -t0.x;
                t0.y = -t0.y;
                t0.z = -t0.z;
                pc += 1;
                continue;
            }
            if (op == kSdfAdd) {   // t1 + t0 -> t0
                if (sp > 1) {
                    t0.v += t1.v;
                    t0.x += t1.x;
                    t0.y += t1.y;
                    t0.z += t1.z;
                    t1 = t2;
                    t2 = t3;
                    if (sp > 4) {
                        t3 = deep[sp - 5];
                    }
                    --sp;
                }
                pc += 1;
                continue;
            }
            if (op == kSdfScale) {
                const float f = sdf_at(g, pc + 1);
                t0.v *= f;
                t0.x *= f;
                t0.y *= f;
                t0.z *= f;
                pc += 2;
                continue;
            }
            SdfV nv = sdf_zero();   // an operand
            if (op == kSdfPrim) {
                const int type = (int)sdf_at(g, pc + 1);
                const int np = sdf_nparam(type);
                if ((int64_t)pc + 2 + np > g.ntw) {
                    break;   // (a malformed program)
                }
                const float* q = g.gTW + pc + 2;
                // the value and (grad) central differences of this primitive
                const float e = fmaxf(1e-4f * (fabsf(q[0]) + fabsf(q[1]) + fabsf(q[2]) + 1.0f), 1e-5f);
                const int ne = grad ? 7 : 1;
                float fv[7];
                for (int k = 0; k < ne; ++k) {
                    const float dd = k == 0 ? 0.0f : ((k & 1) ? e : -e);
                    const int ax = (k - 1) >> 1;
                    fv[k] = sdf_prim(type, q, x + (ax == 0 ? dd : 0.0f), y + (ax == 1 ? dd : 0.0f),
                                     z + (ax == 2 ? dd : 0.0f));
                }
                nv.v = fv[0];
                if (grad) {
                    nv.x = (fv[1] - fv[2]) / (2.0f * e);
                    nv.y = (fv[3] - fv[4]) / (2.0f * e);
                    nv.z = (fv[5] - fv[6]) / (2.0f * e);
                }
                pc += 2 + np;
            } else if (op == kSdfBbox) {
                // culled: far from the object's box its term is a constant bound
                const float lo0 = sdf_at(g, pc + 1), lo1 = sdf_at(g, pc + 2), lo2 = sdf_at(g, pc + 3);
                const float hi0 = sdf_at(g, pc + 4), hi1 = sdf_at(g, pc + 5), hi2 = sdf_at(g, pc + 6);
                if (!(x < lo0 - margin || y < lo1 - margin || z < lo2 - margin || x > hi0 + margin ||
                      y > hi1 + margin || z > hi2 + margin)) {
                    pc += 9;
                    continue;
                }
                nv.v = sdf_at(g, pc + 8) * margin;
                pc += 9 + (int)sdf_at(g, pc + 7);
            } else if (op == kSdfMconst) {
                nv.v = sdf_at(g, pc + 1) * margin;
                pc += 2;
            } else if (op == kSdfConst) {
                nv.v = sdf_at(g, pc + 1);
                pc += 2;
            } else {
                break;   // (a malformed program)
            }
            // an operand followed by a min / max (or NEG then min / max) is
            // combined at once, without the stack's shifts
            {
                const int op1 = (int)sdf_at(g, pc), neg = op1 == kSdfNeg;
                const int op2 = neg ? (int)sdf_at(g, pc + 1) : op1;
                if (sp > 0 && sdf_is_minmax(op2)) {
                    if (neg) {
                        nv.v = -nv.v;
                        nv.x = -nv.x;
                        nv.y = -nv.y;
                        nv.z = -nv.z;
                    }
                    t0 = sdf_minmax(t0, nv, op2 == kSdfMax || op2 == kSdfCmax ? -1.0f : 1.0f, kblend,
                                    op2 >= kSdfCmax ? 0.0f : kgap, grad, &near);
                    pc += 1 + neg;
                    continue;
                }
            }
            if (sp < kSdfStack) {   // push
                if (sp >= 4) {
                    deep[sp - 4] = t3;
                }
                t3 = t2;
                t2 = t1;
                t1 = t0;
                t0 = nv;
                ++sp;
            }
        }
        if (grad || !near) {
            break;
        }
        grad = 1;
    }
    return sp > 0 ? t0 : none;
}

__device__ __forceinline__ float sdf_value(const DGrid& g, int l, float px, float py, float pz) {
    return sdf_evalv(g, l, px, py, pz, 0).v;
}

// phi_l of the analytic fields: clamp(0.5 + s_l / w) (src/opencl/v2m_seed_body.cl:33-37)
__device__ __forceinline__ float sdf_phi(const DGrid& g, int l, float px, float py, float pz) {
    return fminf(1.0f, fmaxf(0.0f, 0.5f + sdf_value(g, l, px, py, pz) / sdf_at(g, 1)));
}

// psi_ab = (s_a - s_b) / w, and (gr) its gradient (src/opencl/v2m_seed_body.cl:182-184, 214-221)
__device__ __forceinline__ float sdf_psi(const DGrid& g, int a, int b, float px, float py, float pz, float* gr) {
    const float w = sdf_at(g, 1);
    if (!gr) {
        return (sdf_value(g, a, px, py, pz) - sdf_value(g, b, px, py, pz)) / w;
    }
    const SdfV sa = sdf_evalv(g, a, px, py, pz, 1), sb = sdf_evalv(g, b, px, py, pz, 1);
    gr[0] = (sa.x - sb.x) / w;
    gr[1] = (sa.y - sb.y) / w;
    gr[2] = (sa.z - sb.z) / w;
    return (sa.v - sb.v) / w;
}

}  // namespace
}  // namespace v2m
