// Feature evaluation at points where the surface is not smooth: exact zeros
// and tied min/max arguments (FeatureEvaluator, libfive/src/eval/
// eval_feature.cpp:56-372, and Feature, libfive/src/eval/feature.cpp:14-284).
//
// These points are rare, so one lane of the warp runs the evaluator serially
// while the others wait.  Its workspace is a per-warp slice of global memory
// (kRegBlock floats per tape register) plus a small per-warp scratch area:
// every register holds up to kMaxFeat features of up to kMaxEps epsilon
// directions.  Capacity overflows are reported through the status
// word (ST_FEATURE_OVERFLOW), never silently truncated.
#pragma once
#include "dc_device.cuh"

namespace lfb {

constexpr int kMaxFeat = 15;         // per register
constexpr int kMaxEps = 4;           // per feature
constexpr int kFeatFloats = 16;      // deriv[3], neps, eps[4][3]
constexpr int kRegBlock = 256;       // floats per register in the workspace
constexpr int kValOff = kMaxFeat * kFeatFloats;          // 240
constexpr int kCountOff = kValOff + 1;                   // 241
static_assert(kCountOff < kRegBlock, "feature lists must fit a register block");
constexpr int kTmpFeat = 64;         // candidate features of one clause
constexpr int kTmpCorners = 168;     // plane triples in Feature::check: C(11, 3) = 165

/// A Feature::check request from the evaluating lane to the whole warp.
struct FeatCheckReq {
    float f[kFeatFloats];
    float e[3];
    int op;                          // FEAT_REQ_CHECK or FEAT_REQ_DONE
    int found1;                      // some vertex is inside
    int found2;                      // some midpoint is inside
};
enum : int { FEAT_REQ_CHECK = 1, FEAT_REQ_DONE = 2 };

struct __align__(16) FeatureScratch {
    float feats[kTmpFeat][kFeatFloats];
    float corners[kTmpCorners][3];   // one slot per plane triple
    float one[2][kFeatFloats];       // constant operands
    FeatCheckReq req;
};

struct FeatCtx {
    float* regs;               // n_regs * kRegBlock floats
    FeatureScratch* tmp;
    uint32_t* status;
};

////////////////////////////////////////////////////////////////////////////////
// Feature (feature.cpp)

__device__ __forceinline__ float fdot(const float* a, const float* b)
{
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

/// Feature::check(e, dup) (feature.cpp:100-245), evaluated by all 32 lanes
/// of a warp together; every lane reads the same request and gets the same
/// answer.  The polytope vertices (one per triple of planes, in the
/// reference's loop order) are spread over the lanes, then the vertex and
/// midpoint tests.  The reference skips exact-duplicate vertices; the
/// answer ("some vertex, or some midpoint of two vertices, lies strictly
/// inside every plane") is the same with or without them, so none are
/// removed here.  Triples with a repeated plane have two equal columns and
/// an exactly zero determinant, so they are not enumerated.
///
/// Every call passes exactly four __syncwarp barriers on every lane, early
/// answers included, so the evaluating lane and the helpers stay paired.
static __device__ __noinline__ bool feat_check_warp(const FeatCtx& C, bool* dup, int lane)
{
    FeatCheckReq* R = &C.tmp->req;
    float f[kFeatFloats], e[3];
    for (int i = 0; i < kFeatFloats; ++i) f[i] = R->f[i];
    for (int i = 0; i < 3; ++i) e[i] = R->e[i];
    __syncwarp();                                   // 1: request read

    const int n = static_cast<int>(f[3]);
    const float* eps = f + 4;
    bool early = false, early_val = false;
    for (int i = 0; i < n && !early; ++i) {
        if (static_cast<double>(fdot(e, eps + 3 * i)) > 1 - 1e-8) {
            if (dup) *dup = true;
            early = true;
            early_val = true;
        }
    }
    if (!early && n == 0) {
        early = true;
        early_val = true;
    }
    if (!early && n == 1) {
        early = true;
        early_val = fdot(e, eps) != -1;
    }

    // Planes: the epsilons (d = 0) and the six faces of a unit cube (d = 1).
    float pn[kMaxEps + 1 + 6][3];
    float pd[kMaxEps + 1 + 6];
    int np = 0, ne = 0, nc = 0;
    float (*corners)[3] = C.tmp->corners;
    auto inside_all = [&](const float* v) {
        for (int s = 0; s < ne; ++s) {
            if (fdot(v, pn[s]) <= 0) return false;
        }
        return true;
    };
    if (!early) {
        for (int i = 0; i < n; ++i) {
            pn[np][0] = eps[3 * i]; pn[np][1] = eps[3 * i + 1]; pn[np][2] = eps[3 * i + 2];
            pd[np++] = 0.0f;
        }
        pn[np][0] = e[0]; pn[np][1] = e[1]; pn[np][2] = e[2];
        pd[np++] = 0.0f;
        ne = np;   // es = epsilons + e
        const float axes[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0},
                                  {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        for (int k = 0; k < 6; ++k) {
            pn[np][0] = axes[k][0]; pn[np][1] = axes[k][1]; pn[np][2] = axes[k][2];
            pd[np++] = 1.0f;
        }
        bool found = false;
        for (int i = 0; i < np; ++i) {
            for (int j = i + 1; j < np; ++j) {
                for (int k = j + 1; k < np; ++k) {
                    if (pd[i] == 0.0f && pd[j] == 0.0f && pd[k] == 0.0f) continue;
                    const int slot = nc++;
                    if ((slot & 31) != lane) continue;
                    // M = [a b c] as columns (Eigen's comma initializer)
                    float m[3][3];
                    for (int r = 0; r < 3; ++r) {
                        m[r][0] = pn[i][r];
                        m[r][1] = pn[j][r];
                        m[r][2] = pn[k][r];
                    }
                    auto det3h = [&](int a, int b, int c) {
                        const float p = m[1][b] * m[2][c];
                        const float q = m[1][c] * m[2][b];
                        return m[0][a] * (p - q);
                    };
                    const float det = (det3h(0, 1, 2) - det3h(1, 0, 2)) + det3h(2, 0, 1);
                    if (static_cast<double>(fabsf(det)) < 1e-6) {
                        corners[slot][0] = LF_QNAN;   // no vertex
                        continue;
                    }
                    auto cof = [&](int i_, int j_) {
                        const int i1 = (i_ + 1) % 3, i2 = (i_ + 2) % 3;
                        const int j1 = (j_ + 1) % 3, j2 = (j_ + 2) % 3;
                        const float p = m[i1][j1] * m[i2][j2];
                        const float q = m[i1][j2] * m[i2][j1];
                        return p - q;
                    };
                    const float c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
                    const float dd = (c00 * m[0][0] + c10 * m[1][0]) + c20 * m[2][0];
                    const float inv = 1.0f / dd;
                    float mi[3][3];
                    for (int jj = 0; jj < 3; ++jj) {
                        for (int ii = 0; ii < 3; ++ii) mi[ii][jj] = cof(jj, ii) * inv;
                    }
                    const float dv[3] = {pd[i], pd[j], pd[k]};
                    float v[3];
                    for (int r = 0; r < 3; ++r) {
                        const float p0 = mi[r][0] * dv[0], p1 = mi[r][1] * dv[1],
                                    p2 = mi[r][2] * dv[2];
                        v[r] = (p0 + p1) + p2;
                    }
                    corners[slot][0] = v[0]; corners[slot][1] = v[1]; corners[slot][2] = v[2];
                    found |= inside_all(v);
                }
            }
        }
        if (found) R->found1 = 1;
    }
    __syncwarp();                                   // 2: vertices written
    const bool any1 = !early && R->found1 != 0;
    if (!early && !any1) {
        bool found = false;
        for (int pq = lane; pq < nc * nc && !found; pq += 32) {
            const int q = pq / nc, w = pq - q * nc;
            const float* cq = corners[q];
            const float* cw = corners[w];
            if (cq[0] != cq[0] || cw[0] != cw[0]) continue;
            float p[3];
            for (int r = 0; r < 3; ++r) p[r] = (cq[r] + cw[r]) / 2.0f;
            found = inside_all(p);
        }
        if (found) R->found2 = 1;
    }
    __syncwarp();                                   // 3: midpoints tested
    const bool any2 = R->found2 != 0;
    __syncwarp();                                   // 4: flags read
    return early ? early_val : (any1 || any2);
}

/// Feature::check from the evaluating lane (lane 0): posts the request and
/// joins the other lanes, which wait in feat_serve.
__device__ inline bool feat_check(const FeatCtx& C, const float* f, const float* e,
                                  bool* dup)
{
    FeatCheckReq* R = &C.tmp->req;
    for (int i = 0; i < kFeatFloats; ++i) R->f[i] = f[i];
    R->e[0] = e[0]; R->e[1] = e[1]; R->e[2] = e[2];
    R->found1 = 0;
    R->found2 = 0;
    R->op = FEAT_REQ_CHECK;
    __syncwarp();
    return feat_check_warp(C, dup, 0);
}

/// The other lanes' side of feat_check, until lane 0 posts FEAT_REQ_DONE.
__device__ inline void feat_serve(const FeatCtx& C, int lane)
{
    FeatCheckReq* R = &C.tmp->req;
    while (true) {
        __syncwarp();
        if (*reinterpret_cast<volatile int*>(&R->op) == FEAT_REQ_DONE) break;
        feat_check_warp(C, nullptr, lane);
    }
}

/// Ends lane 0's side of a warp-collective feature evaluation.
__device__ inline void feat_done(const FeatCtx& C)
{
    C.tmp->req.op = FEAT_REQ_DONE;
    __syncwarp();
}

/// Feature::push(e) (feature.cpp:50-72).
__device__ inline bool feat_push(const FeatCtx& C, float* f, const float* e_)
{
    const float nrm = sqrtf(fdot(e_, e_));
    if (nrm == 0) return false;
    const float e[3] = {e_[0] / nrm, e_[1] / nrm, e_[2] / nrm};
    bool dup = false;
    if (feat_check(C, f, e, &dup)) {
        if (!dup) {
            const int n = static_cast<int>(f[3]);
            if (n >= kMaxEps) {
                atomicOr(C.status, ST_FEATURE_OVERFLOW | ST_FEAT_EPS);
                return false;
            }
            f[4 + 3 * n] = e[0]; f[5 + 3 * n] = e[1]; f[6 + 3 * n] = e[2];
            f[3] = static_cast<float>(n + 1);
        }
        return true;
    }
    return false;
}

__device__ __forceinline__ int vcmp3(const float* a, const float* b)
{
    for (int i = 0; i < 3; ++i) {
        if (a[i] < b[i]) return -1;
        if (a[i] > b[i]) return 1;
    }
    return 0;
}

/// Feature::operator< (feature.cpp:247-284).
__device__ __forceinline__ bool feat_less(const float* a, const float* b)
{
    const int na = static_cast<int>(a[3]), nb = static_cast<int>(b[3]);
    int i = 0;
    for (; i < na && i < nb; ++i) {
        const int c = vcmp3(a + 4 + 3 * i, b + 4 + 3 * i);
        if (c != 0) return c < 0;
    }
    if (i < na) return false;
    if (i < nb) return true;
    return vcmp3(a, b) < 0;
}

__device__ __forceinline__ bool feat_same_eps(const float* a, const float* b)
{
    if (a[3] != b[3]) return false;
    const int n = static_cast<int>(a[3]);
    for (int i = 0; i < 3 * n; ++i) {
        if (a[4 + i] != b[4 + i]) return false;
    }
    return true;
}

/// Copies one feature (both pointers 16-byte aligned).
__device__ __forceinline__ void feat_copy(float* dst, const float* src)
{
    const float4* s = reinterpret_cast<const float4*>(src);
    float4* d = reinterpret_cast<float4*>(dst);
    const float4 a = s[0], b = s[1], c = s[2], e = s[3];
    d[0] = a; d[1] = b; d[2] = c; d[3] = e;
}

/// One feature held in registers (all indices static after unrolling).
struct FeatReg {
    float v[kFeatFloats];
};

__device__ __forceinline__ FeatReg feat_get(const float* src)
{
    FeatReg r;
    const float4* s = reinterpret_cast<const float4*>(src);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float4 q = s[i];
        r.v[4 * i] = q.x; r.v[4 * i + 1] = q.y; r.v[4 * i + 2] = q.z; r.v[4 * i + 3] = q.w;
    }
    return r;
}

__device__ __forceinline__ void feat_put(float* dst, const FeatReg& r)
{
    float4* d = reinterpret_cast<float4*>(dst);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        d[i] = make_float4(r.v[4 * i], r.v[4 * i + 1], r.v[4 * i + 2], r.v[4 * i + 3]);
    }
}

////////////////////////////////////////////////////////////////////////////////
// FeatureEvaluator::operator() (eval_feature.cpp:171-372) over a register tape

static __device__ __noinline__ void feat_eval(const FeatCtx& C, const DevTape& bt,
                                 const RegClause* cl, uint32_t len, float x,
                                 float y, float z, float* root_val,
                                 const float** root_list, int* root_n)
{
    float* W = C.regs;
    const float in[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
        float* b = W + a * kRegBlock;
        for (int i = 0; i < kFeatFloats; ++i) b[i] = 0.0f;
        b[a] = 1.0f;
        b[kValOff] = in[a];
        b[kCountOff] = 1.0f;
    }
    FeatureScratch* T = C.tmp;
    for (int i = 0; i < kFeatFloats; ++i) {
        T->one[0][i] = 0.0f;
        T->one[1][i] = 0.0f;
    }
    uint2 next = len ? __ldg(reinterpret_cast<const uint2*>(cl)) : make_uint2(0, 0);
    for (uint32_t c = 0; c < len; ++c) {
        const uint2 raw = next;
        if (c + 1 < len) next = __ldg(reinterpret_cast<const uint2*>(cl + c + 1));
        const uint8_t o = raw.x & 0xff;
        const uint8_t kinds = (raw.x >> 8) & 0xff;
        const uint16_t ro = raw.x >> 16;
        const bool binary = dev_is_binary(o);

        // Plain fast path: operands with one feature and no epsilons (a
        // plain value and gradient) and no tied min/max give a plain
        // result, the clause's ordinary derivative; this is what the
        // general path below computes for them.
        {
            float4 ga = make_float4(0.0f, 0.0f, 0.0f, 0.0f), gb = ga;
            float2 va, vb = make_float2(0.0f, 1.0f);
            const uint16_t ia = raw.y & 0xffff, ib = raw.y >> 16;
            if ((kinds & 3) == OPND_REG) {
                ga = *reinterpret_cast<const float4*>(W + ia * kRegBlock);
                va = *reinterpret_cast<const float2*>(W + ia * kRegBlock + kValOff);
            } else {
                va = make_float2(__ldg(bt.cpool + ia), 1.0f);
            }
            if (binary) {
                if (((kinds >> 2) & 3) == OPND_REG) {
                    gb = *reinterpret_cast<const float4*>(W + ib * kRegBlock);
                    vb = *reinterpret_cast<const float2*>(W + ib * kRegBlock + kValOff);
                } else {
                    vb = make_float2(__ldg(bt.cpool + ib), 1.0f);
                }
            }
            const bool plain = va.y == 1.0f && ga.w == 0.0f &&
                               (!binary || (vb.y == 1.0f && gb.w == 0.0f));
            const bool tie = (o == op::MIN || o == op::MAX) && va.x == vb.x;
            if (plain && !tie) {
                const D4 r = dv_deriv(o, D4{va.x, ga.x, ga.y, ga.z}, D4{vb.x, gb.x, gb.y, gb.z},
                                      false);
                float* out = W + ro * kRegBlock;
                *reinterpret_cast<float4*>(out) = make_float4(r.dx, r.dy, r.dz, 0.0f);
                *reinterpret_cast<float2*>(out + kValOff) = make_float2(r.v, 1.0f);
                continue;
            }
        }
        float av, bv = 0.0f;
        const float* fa;
        const float* fb = T->one[1];
        int na, nb = 1;
        {
            const uint16_t ia = raw.y & 0xffff;
            if ((kinds & 3) == OPND_REG) {
                const float* b = W + ia * kRegBlock;
                av = b[kValOff]; fa = b; na = static_cast<int>(b[kCountOff]);
            } else {
                av = __ldg(bt.cpool + ia); fa = T->one[0]; na = 1;
            }
        }
        if (binary) {
            const uint16_t ib = raw.y >> 16;
            if (((kinds >> 2) & 3) == OPND_REG) {
                const float* b = W + ib * kRegBlock;
                bv = b[kValOff]; fb = b; nb = static_cast<int>(b[kCountOff]);
            } else {
                bv = __ldg(bt.cpool + ib); fb = T->one[1]; nb = 1;
            }
        }
        const float ov = dv_value(o, av, bv);
        float* out = W + ro * kRegBlock;

        // Fast paths (the result needs no sorting or merging): a min/max
        // whose arguments differ or a copy passes one operand's list on; a
        // clause over single features gives a single feature.  The general
        // path below produces the same lists for these cases.
        {
            const float* src = nullptr;
            int ns = 0;
            if ((o == op::MIN || o == op::MAX) && av != bv) {
                const bool take_a = (o == op::MIN) == (av < bv);
                src = take_a ? fa : fb;
                ns = take_a ? na : nb;
            } else if (o == OP_COPY) {
                src = fa;
                ns = na;
            }
            if (src) {
                if (src != out) {
                    for (int i = 0; i < ns; ++i) {
                        feat_copy(out + i * kFeatFloats, src + i * kFeatFloats);
                    }
                }
                out[kValOff] = ov;
                out[kCountOff] = static_cast<float>(ns);
                continue;
            }
            if (na == 1 && (!binary || (nb == 1 && o != op::MIN && o != op::MAX))) {
                FeatReg d = feat_get(fa);
                const D4 r = binary ? dv_deriv(o, D4{av, d.v[0], d.v[1], d.v[2]},
                                               D4{bv, fb[0], fb[1], fb[2]}, false)
                                    : dv_deriv(o, D4{av, d.v[0], d.v[1], d.v[2]},
                                               D4{0, 0, 0, 0}, false);
                d.v[0] = r.dx; d.v[1] = r.dy; d.v[2] = r.dz;
                if (binary && fb[3] != 0.0f) {
                    // Merge B's epsilons, skipping exact duplicates.
                    const FeatReg B = feat_get(fb);
                    const int nbe = static_cast<int>(B.v[3]);
                    int n = static_cast<int>(d.v[3]);
#pragma unroll
                    for (int q = 0; q < kMaxEps; ++q) {
                        if (q >= nbe) break;
                        const float e0 = B.v[4 + 3 * q], e1 = B.v[5 + 3 * q], e2 = B.v[6 + 3 * q];
                        bool found = false;
#pragma unroll
                        for (int w = 0; w < kMaxEps; ++w) {
                            // vcmp3(e, eps_w) == 0: no component orders either way
                            found |= w < n && !(e0 < d.v[4 + 3 * w]) && !(e0 > d.v[4 + 3 * w]) &&
                                     !(e1 < d.v[5 + 3 * w]) && !(e1 > d.v[5 + 3 * w]) &&
                                     !(e2 < d.v[6 + 3 * w]) && !(e2 > d.v[6 + 3 * w]);
                        }
                        if (found) continue;
                        if (n >= kMaxEps) {
                            atomicOr(C.status, ST_FEATURE_OVERFLOW | ST_FEAT_EPS);
                            break;
                        }
#pragma unroll
                        for (int w = 0; w < kMaxEps; ++w) {
                            if (w == n) {
                                d.v[4 + 3 * w] = e0; d.v[5 + 3 * w] = e1; d.v[6 + 3 * w] = e2;
                            }
                        }
                        ++n;
                        d.v[3] = static_cast<float>(n);
                    }
                }
                feat_put(out, d);
                out[kValOff] = ov;
                out[kCountOff] = 1.0f;
                continue;
            }
        }

        int nt = 0;
        bool overflow = false, tmp_over = false;
        auto emit = [&](const float* f) -> float* {
            if (nt >= kTmpFeat) {
                tmp_over = true;
                return nullptr;
            }
            float* d = T->feats[nt++];
            feat_copy(d, f);
            return d;
        };
        if (o == op::MIN || o == op::MAX) {
            const bool is_min = o == op::MIN;
            if (av < bv) {
                const float* src = is_min ? fa : fb;
                const int ns = is_min ? na : nb;
                for (int i = 0; i < ns; ++i) emit(src + i * kFeatFloats);
            } else if (av > bv) {
                const float* src = is_min ? fb : fa;
                const int ns = is_min ? nb : na;
                for (int i = 0; i < ns; ++i) emit(src + i * kFeatFloats);
            } else {
                for (int i = 0; i < na; ++i) {
                    const float* A = fa + i * kFeatFloats;
                    for (int j = 0; j < nb; ++j) {
                        const float* B = fb + j * kFeatFloats;
                        float eps[3];
                        for (int k = 0; k < 3; ++k) {
                            eps[k] = is_min ? B[k] - A[k] : A[k] - B[k];
                        }
                        if (sqrtf(fdot(eps, eps)) == 0) {
                            if (A[3] != 0) emit(A);
                            if (B[3] != 0) emit(B);
                            if (A[3] == 0 && B[3] == 0) emit(A);
                        } else {
                            // combined = A with B's epsilons pushed
                            __align__(16) float comb[kFeatFloats];
                            feat_copy(comb, A);
                            bool ok = true;
                            const int nbe = static_cast<int>(B[3]);
                            for (int q = 0; q < nbe && ok; ++q) ok = feat_push(C, comb, B + 4 + 3 * q);
                            if (ok) {
                                __align__(16) float fa2[kFeatFloats];
                                feat_copy(fa2, comb);
                                fa2[0] = A[0]; fa2[1] = A[1]; fa2[2] = A[2];
                                if (feat_push(C, fa2, eps)) emit(fa2);
                                __align__(16) float fb2[kFeatFloats];
                                feat_copy(fb2, comb);
                                fb2[0] = B[0]; fb2[1] = B[1]; fb2[2] = B[2];
                                const float neg[3] = {-eps[0], -eps[1], -eps[2]};
                                if (feat_push(C, fb2, neg)) emit(fb2);
                            }
                        }
                    }
                }
            }
        } else if (o == OP_COPY) {
            for (int i = 0; i < na; ++i) emit(fa + i * kFeatFloats);
        } else if (!binary) {
            for (int i = 0; i < na; ++i) {
                const float* A = fa + i * kFeatFloats;
                const D4 r = dv_deriv(o, D4{av, A[0], A[1], A[2]}, D4{0, 0, 0, 0}, false);
                float* d = emit(A);
                if (d) { d[0] = r.dx; d[1] = r.dy; d[2] = r.dz; }
            }
        } else {
            for (int i = 0; i < na; ++i) {
                const float* A = fa + i * kFeatFloats;
                for (int j = 0; j < nb; ++j) {
                    const float* B = fb + j * kFeatFloats;
                    const D4 r = dv_deriv(o, D4{av, A[0], A[1], A[2]},
                                          D4{bv, B[0], B[1], B[2]}, false);
                    float* d = emit(A);
                    if (!d) continue;
                    d[0] = r.dx; d[1] = r.dy; d[2] = r.dz;
                    // merge B's epsilons, skipping exact duplicates
                    const int nbe = static_cast<int>(B[3]);
                    for (int q = 0; q < nbe; ++q) {
                        const float* e = B + 4 + 3 * q;
                        const int n = static_cast<int>(d[3]);
                        bool found = false;
                        for (int w = 0; w < n && !found; ++w) found = vcmp3(e, d + 4 + 3 * w) == 0;
                        if (found) continue;
                        if (n >= kMaxEps) {
                            overflow = true;
                            break;
                        }
                        d[4 + 3 * n] = e[0]; d[5 + 3 * n] = e[1]; d[6 + 3 * n] = e[2];
                        d[3] = static_cast<float>(n + 1);
                    }
                }
            }
        }
        // Deduplicate: sort, drop near-duplicates with equal epsilons, and
        // collapse to one plain feature if all gradients agree.
        if (nt > 1) {
            for (int i = 1; i < nt; ++i) {
                __align__(16) float cur[kFeatFloats];
                feat_copy(cur, T->feats[i]);
                int j = i - 1;
                while (j >= 0 && feat_less(cur, T->feats[j])) {
                    feat_copy(T->feats[j + 1], T->feats[j]);
                    --j;
                }
                feat_copy(T->feats[j + 1], cur);
            }
            int m = 1;
            for (int i = 1; i < nt; ++i) {
                const float* last = T->feats[m - 1];
                const float* f = T->feats[i];
                const float dd[3] = {f[0] - last[0], f[1] - last[1], f[2] - last[2]};
                if (static_cast<double>(fdot(dd, dd)) <= 1e-10 && feat_same_eps(f, last)) {
                    continue;
                }
                if (m != i) feat_copy(T->feats[m], f);
                ++m;
            }
            nt = m;
            bool all_same = true;
            for (int i = 0; i < nt && all_same; ++i) {
                const float dd[3] = {T->feats[i][0] - T->feats[0][0],
                                     T->feats[i][1] - T->feats[0][1],
                                     T->feats[i][2] - T->feats[0][2]};
                all_same = static_cast<double>(fdot(dd, dd)) < 1e-10;
            }
            if (all_same) {
                T->feats[0][3] = 0.0f;
                nt = 1;
            }
        }
        if (nt > kMaxFeat || overflow || tmp_over) {
            atomicOr(C.status, ST_FEATURE_OVERFLOW | (overflow ? ST_FEAT_EPS : 0u) |
                                   (tmp_over ? ST_FEAT_TMP : 0u) |
                                   (nt > kMaxFeat ? ST_FEAT_LIST : 0u));
            if (nt > kMaxFeat) nt = kMaxFeat;
        }
        for (int i = 0; i < nt; ++i) feat_copy(out + i * kFeatFloats, T->feats[i]);
        out[kValOff] = ov;
        out[kCountOff] = static_cast<float>(nt);
    }
    if (bt.root_kind == OPND_REG) {
        const float* b = W + bt.root * kRegBlock;
        *root_val = b[kValOff];
        *root_list = b;
        *root_n = static_cast<int>(b[kCountOff]);
    } else {
        *root_val = __ldg(bt.cpool + bt.root);
        *root_list = T->one[0];
        *root_n = 1;
    }
}

/// FeatureEvaluator::isInside (eval_feature.cpp:56-116).  Warp-collective:
/// every lane passes the same point.
static __device__ __noinline__ bool dev_is_inside(const FeatCtx& C, const DevTape& bt,
                                     const RegClause* cl, uint32_t len, float x,
                                     float y, float z, int lane)
{
    int inside = 0;
    __syncwarp();
    if (lane == 0) {
        float v;
        const float* fs;
        int n;
        feat_eval(C, bt, cl, len, x, y, z, &v, &fs, &n);
        if (v < 0) {
            inside = 1;
        } else if (v > 0) {
            inside = 0;
        } else if (n == 1) {
            inside = sqrtf(fdot(fs, fs)) > 0;
        } else {
            bool pos = false, neg = false;
            for (int i = 0; i < n; ++i) {
                const float* f = fs + i * kFeatFloats;
                const float nd[3] = {-f[0], -f[1], -f[2]};
                pos |= feat_check(C, f, f, nullptr);
                neg |= feat_check(C, f, nd, nullptr);
            }
            inside = !(pos && !neg);
        }
        feat_done(C);
    } else {
        feat_serve(C, lane);
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, inside, 0) != 0;
}

/// One QEF sample per distinct feature gradient (dc_tree.inl:456-469 with
/// FeatureEvaluator::features, eval_feature.cpp:151-169).  Warp-collective.
static __device__ __noinline__ void dev_push_features(const FeatCtx& C, const DevTape& bt,
                                         const RegClause* cl, uint32_t len,
                                         const double pos[3], double value,
                                         Qef* q, uint8_t* exists, int lane)
{
    __syncwarp();
    if (lane == 0) {
        float v;
        const float* fs;
        int n;
        feat_eval(C, bt, cl, len, static_cast<float>(pos[0]),
                  static_cast<float>(pos[1]), static_cast<float>(pos[2]), &v, &fs, &n);
        for (int i = 0; i < n; ++i) {
            const float* f = fs + i * kFeatFloats;
            bool seen = false;
            for (int j = 0; j < i && !seen; ++j) seen = vcmp3(f, fs + j * kFeatFloats) == 0;
            if (seen) continue;
            const double g[3] = {f[0], f[1], f[2]};
            qef_push(*q, pos, g, value);
            *exists = 1;
        }
        feat_done(C);
    } else {
        feat_serve(C, lane);
    }
    __syncwarp();
}

}  // namespace lfb
