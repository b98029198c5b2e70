// Docking engine kernels for sm_100a.
//
//  * maps_kernel      receptor grid maps (one thread per grid point, all
//                     requested types at once, receptor atoms of the tile staged
//                     in shared memory in index order)
//  * score_kernel     energy + pose gradient at fixed poses (one warp per pose)
//  * optimize_kernel  BFGS local optimisation from given poses (one warp per pose)
//  * search_kernel    Monte-Carlo + BFGS chains (one warp per chain), plain fixed
//                     tiling or a persistent queue over (ligand, chain) items
//
// A chain's state (conformations, gradients, inverse Hessian, atom
// coordinates, forces, node frames) lives in shared memory; ligand topology is
// read through the read-only cache; grid maps and pair tables stay L2-resident.
// The search kernel is one flat loop around a single energy evaluation with a
// warp-uniform state machine for the BFGS line search and the Monte-Carlo
// steps, so the evaluation code exists once and the chain context stays in
// registers.  Per-evaluation arithmetic follows the reference's
// model::eval_deriv (unidock/src/lib/model.cpp:935-962): forward kinematics
// (tree.h:89-128), trilinear grid energy/gradient with out-of-box penalty
// (grid.cpp:40-129), lerped pair tables (precalculate.h:48-65), curl
// (curl.h:28-43) and the force/torque sums up the torsion tree
// (tree.h:75-84,164-192).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <unordered_map>

#include "ud_engine.h"

namespace ud {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;
constexpr float kPi = 3.1415926535897931f;
constexpr float kEps = 1.1920928955078125e-07f;  // FLT_EPSILON
constexpr float kMaxFl = 3.402823466e+38f;

// ---------------------------------------------------------------- RNG
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011).
struct Philox {
    uint32_t k0, k1;   // key (seed)
    uint32_t c0, c1, c2, c3;
    __device__ void init(unsigned long long seed, uint32_t stream, uint32_t sub) {
        k0 = (uint32_t)seed;
        k1 = (uint32_t)(seed >> 32);
        c0 = 0; c1 = 0; c2 = stream; c3 = sub;
    }
    // out of line: only lane 0 draws, and inlining 10 rounds at every call
    // site would grow the hot loop's code footprint
    __device__ __noinline__ uint4 next() {
        uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3, a = k0, b = k1;
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            uint32_t hi0 = __umulhi(0xD2511F53u, x0), lo0 = 0xD2511F53u * x0;
            uint32_t hi1 = __umulhi(0xCD9E8D57u, x2), lo1 = 0xCD9E8D57u * x2;
            uint32_t n0 = hi1 ^ x1 ^ a, n2 = hi0 ^ x3 ^ b;
            x0 = n0; x1 = lo1; x2 = n2; x3 = lo0;
            a += 0x9E3779B9u;
            b += 0xBB67AE85u;
        }
        if (++c0 == 0) ++c1;
        return make_uint4(x0, x1, x2, x3);
    }
};
__device__ __forceinline__ float u01(uint32_t u) { return (u >> 8) * (1.0f / 16777216.0f); }

// ---------------------------------------------------------------- math
// normalize_angle of unidock/src/lib/common.h:252-270 (values within
// [-3 pi, 3 pi] take one step; larger ones the ceil formula first).
__device__ __forceinline__ float normalized_angle(float x) {
    if (x > 3 * kPi) x -= 2 * kPi * ceilf((x - kPi) / (2 * kPi));
    else if (x < -3 * kPi) x += 2 * kPi * ceilf((-x - kPi) / (2 * kPi));
    if (x > kPi) x -= 2 * kPi;
    else if (x < -kPi) x += 2 * kPi;
    return x;
}

__device__ __forceinline__ void qmul(const float* a, const float* b, float* o) {
    float t0 = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    float t1 = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    float t2 = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
    float t3 = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
    o[0] = t0; o[1] = t1; o[2] = t2; o[3] = t3;
}

__device__ __forceinline__ void qnormalize_approx(float* q) {
    float s = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (fabsf(s - 1) >= 1e-6f) {
        float inv = rsqrtf(s);
        q[0] *= inv; q[1] *= inv; q[2] *= inv; q[3] *= inv;
    }
}

// sin and cos of h in [-pi/2, pi/2] by their Taylor series to the x^15 / x^14
// terms (truncation error below 1e-9 at |h| = pi/2), evaluated with Horner's
// rule; no range reduction is needed because callers pass half angles of
// normalised angles.
__device__ __forceinline__ void sincos_half(float h, float* s, float* c) {
    const float x2 = h * h;
    float ps = -1.0f / 1307674368000.0f;              // -1/15!
    ps = fmaf(ps, x2, 1.0f / 6227020800.0f);          //  1/13!
    ps = fmaf(ps, x2, -1.0f / 39916800.0f);           // -1/11!
    ps = fmaf(ps, x2, 1.0f / 362880.0f);              //  1/9!
    ps = fmaf(ps, x2, -1.0f / 5040.0f);               // -1/7!
    ps = fmaf(ps, x2, 1.0f / 120.0f);                 //  1/5!
    ps = fmaf(ps, x2, -1.0f / 6.0f);                  // -1/3!
    *s = fmaf(ps * x2, h, h);
    float pc = -1.0f / 87178291200.0f;                // -1/14!
    pc = fmaf(pc, x2, 1.0f / 479001600.0f);           //  1/12!
    pc = fmaf(pc, x2, -1.0f / 3628800.0f);            // -1/10!
    pc = fmaf(pc, x2, 1.0f / 40320.0f);               //  1/8!
    pc = fmaf(pc, x2, -1.0f / 720.0f);                // -1/6!
    pc = fmaf(pc, x2, 1.0f / 24.0f);                  //  1/4!
    pc = fmaf(pc, x2, -0.5f);                         // -1/2!
    *c = fmaf(pc, x2, 1.0f);
}

__device__ __forceinline__ void axis_angle_q(const float* axis, float angle, float* q) {
    angle = normalized_angle(angle);
    float s, c;
    sincos_half(0.5f * angle, &s, &c);
    q[0] = c; q[1] = s * axis[0]; q[2] = s * axis[1]; q[3] = s * axis[2];
}

// q <- angle_to_quaternion(rotation) * q, normalised (quaternion.cpp:116-132)
__device__ __forceinline__ void quaternion_increment(float* q, const float* rot) {
    float angle = sqrtf(rot[0] * rot[0] + rot[1] * rot[1] + rot[2] * rot[2]);
    float t[4] = {1, 0, 0, 0};
    if (angle > kEps) {
        const float inv = __frcp_rn(angle);
        float ax[3] = {rot[0] * inv, rot[1] * inv, rot[2] * inv};
        axis_angle_q(ax, angle, t);
    }
    float o[4];
    qmul(t, q, o);
    qnormalize_approx(o);
    q[0] = o[0]; q[1] = o[1]; q[2] = o[2]; q[3] = o[3];
}

// Row-major rotation matrix of quaternion_to_r3 (quaternion.cpp:84-115)
__device__ __forceinline__ void q_to_r3(const float* q, float* m) {
    float a = q[0], b = q[1], c = q[2], d = q[3];
    float aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c, bd = b * d,
          cc = c * c, cd = c * d, dd = d * d;
    m[0] = aa + bb - cc - dd; m[1] = 2 * (-ad + bc); m[2] = 2 * (ac + bd);
    m[3] = 2 * (ad + bc); m[4] = aa - bb + cc - dd; m[5] = 2 * (-ab + cd);
    m[6] = 2 * (-ac + bd); m[7] = 2 * (ab + cd); m[8] = aa - bb - cc + dd;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// A chain runs on kW lanes: the whole warp (32) or one half of it (16), the
// two halves of a warp then being two independent chains.  Masks, sums and
// barriers below involve only the calling chain's lanes.
template <int kW>
__device__ __forceinline__ unsigned lanes_mask() {
    static_assert(kW == 32 || kW == 16, "a chain spans a warp or half a warp");
    if constexpr (kW == 32) return kFull;
    else return 0xFFFFu << (threadIdx.x & 16);
}

template <int kW>
__device__ __forceinline__ float lanes_sum(float v) {
    const unsigned m = lanes_mask<kW>();
#pragma unroll
    for (int o = kW / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
    return v;
}

// Two or three sums at once: the same shuffle tree per value, interleaved so
// that one reduction's latency covers all of them.
template <int kW>
__device__ __forceinline__ void lanes_sum2(float& a, float& b) {
    const unsigned m = lanes_mask<kW>();
#pragma unroll
    for (int o = kW / 2; o > 0; o >>= 1) {
        const float ta = __shfl_xor_sync(m, a, o), tb = __shfl_xor_sync(m, b, o);
        a += ta;
        b += tb;
    }
}
template <int kW>
__device__ __forceinline__ void lanes_sum3(float& a, float& b, float& c) {
    const unsigned m = lanes_mask<kW>();
#pragma unroll
    for (int o = kW / 2; o > 0; o >>= 1) {
        const float ta = __shfl_xor_sync(m, a, o), tb = __shfl_xor_sync(m, b, o), tc = __shfl_xor_sync(m, c, o);
        a += ta;
        b += tb;
        c += tc;
    }
}

template <int kW>
__device__ __forceinline__ void lanes_sync() { __syncwarp(lanes_mask<kW>()); }

// ---------------------------------------------------------------- data views
struct Batch {
    const LigDesc* ligs;
    const AtomRec* atoms;
    const NodeRec* nodes;
    const uint32_t* pairs;
    const uint32_t* grid_list;
    const float* charges;    // AD4: per atom
    const float2* pair_coef; // AD4: per pair slot (q_a q_b, |q_a| V_b + |q_b| V_a)
};

// pair groups whose table rows are in flight together (larger values unroll
// more code into the hot loop, which costs more in instruction fetch than the
// extra loads in flight gain)
#ifndef UD_PAIR_BATCH
#define UD_PAIR_BATCH 1
#endif
constexpr int kPairBatch = UD_PAIR_BATCH;

// Loads of the L2-resident maps and pair tables: read once per use with little
// reuse in L1, so with UD_NA_LOADS they do not allocate L1 lines
// (ld.global.nc.L1::no_allocate), leaving L1 to the ligand topology.
#ifndef UD_NA_LOADS
#define UD_NA_LOADS 1
#endif
#ifndef UD_PAIR_PREFETCH
#define UD_PAIR_PREFETCH 1
#endif
// UD_FORCE_SPLIT (1 or 2): the number of per-atom pair-force arrays; lane
// range r of a pair window adds into array r % UD_FORCE_SPLIT, so that two
// ranges add their forces at once (half the read-modify-write passes)
#ifndef UD_FORCE_SPLIT
#define UD_FORCE_SPLIT 2
#endif
static_assert(UD_FORCE_SPLIT == 1 || UD_FORCE_SPLIT == 2, "1 or 2 force arrays");
// UD_STAGE_ATOMS: each chain copies its ligand's atom records and grid-atom
// words into shared memory at chain start instead of reading them through
// the read-only cache every evaluation
#ifndef UD_STAGE_ATOMS
#define UD_STAGE_ATOMS 1
#endif
// UD_PAIR_PIPE: pair windows software-pipelined one table row ahead
// (UD_PAIR_PIPE_AD4: the AD4 instantiation too, with its E and G rows)
#ifndef UD_PAIR_PIPE
#define UD_PAIR_PIPE 1
#endif
#ifndef UD_PAIR_PIPE_AD4
#define UD_PAIR_PIPE_AD4 1
#endif
__device__ __forceinline__ float2 ld_stream2(const float2* p) {
#if UD_NA_LOADS
    float2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
#else
    return __ldg(p);
#endif
}
__device__ __forceinline__ float4 ld_stream4(const float4* p) {
#if UD_NA_LOADS
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
    return v;
#else
    return __ldg(p);
#endif
}

struct Tables {
    const float4* smooth4; // [tp][bin] (e, dE/dr / r) of bin and bin + 1
    const float* fast;     // [tp][bin]
    int n_bins;
    float factor;
    float cutoff2;
};

// AD4 pair-table rows scaled per pair: electrostatics and charge-dependent
// desolvation (after the AD type-pair rows)
constexpr int kAd4RowE = kAd4TableRowElec, kAd4RowG = kAd4TableRowDesolv;

struct Maps {
    const float* data;     // [slot][z][y][x]
    const float2* xp;      // [slot][z][y][x] = (data at x, data at x + 1): corner pairs in one 8-byte load
    int nx, ny, nz;
    float init[3], factor[3], factor_inv[3], dim_m1[3];
    float slope;
    float corner2[3];
    int e_slot, d_slot;    // AD4: electrostatic and desolvation maps
};

// Receptor atoms in box cells (the device form of DeviceReceptorView).
struct Receptor {
    const float4* atoms;
    const int* start;
    int n[3];
    float begin[3], end[3];
    float inv_cell;
    const BiasRec* bias;
    int n_bias;
    const BiasRec* lig_bias;
    const int* lig_bias_span;
};

// Shared-memory layout of one chain (float offsets).
struct Layout {
    int x, xnew, xorig, tmp, cand, best;
    int g, gnew, gorig, p, y, mhy;
    int h;                 // inverse Hessian, full symmetric n x n (n = 6 + T)
    int coords, forces;
    int frames;
    int prefix;            // per-atom prefix sums of force and moment (6 floats)
    int forces2;           // second pair-force array (float4 per atom) inside the prefix area
    int atomrec;           // the ligand's AtomRec records (4 words per atom), staged at chain start
    int gridl;             // the ligand's grid-atom words (atom | slot << 8), staged at chain start
    int misc;
    int total;
};

__host__ __device__ inline int pad4(int v) { return (v + 3) & ~3; }

__host__ inline Layout make_layout(int max_atoms, int max_tors) {
    Layout L;
    int cs = 7 + max_tors, gs = 6 + max_tors, R = max_tors + 1;
    int o = 0;
    auto take = [&](int n) { int r = o; o += pad4(n); return r; };
    L.x = take(cs); L.xnew = take(cs); L.xorig = take(cs); L.tmp = take(cs); L.cand = take(cs);
    L.best = take(cs);
    L.g = take(gs); L.gnew = take(gs); L.gorig = take(gs); L.p = take(gs); L.y = take(gs);
    L.mhy = take(gs);
    L.h = take(gs * gs);
    L.coords = take(4 * max_atoms);   // float4 per atom (x, y, z, unused)
    L.forces = take(4 * max_atoms);
    L.frames = take(20 * R);
    L.prefix = take(6 * max_atoms);
    // floats [pad4(2A), pad4(2A) + 4A) of the prefix area (A = max_atoms): an
    // iteration of the prefix scan over atoms [base, base + W) reads the
    // second forces of its atoms before its shuffles and writes prefix entries
    // after them, and the entries written so far end at float 6 (base + W),
    // at or below 2A + 4 (base + W) where the next iteration's reads begin
    // (base + W <= A whenever a next iteration exists)
    L.forces2 = L.prefix + pad4(2 * max_atoms);
    L.atomrec = take(UD_STAGE_ATOMS ? 4 * max_atoms : 0);
    L.gridl = take(UD_STAGE_ATOMS ? max_atoms : 0);
    L.misc = take(32);
    L.total = o;
    return L;
}

// Per-warp context of the ligand being worked on (kept in registers): the
// ligand's offsets into the batch arrays, which stay in the kernel parameters
// (a pointer to them costs no register once inlined), rather than seven
// 64-bit pointers.
struct Ctx {
    float* s;              // shared memory of this warp
    const Batch* B;
    int atom_off, node_off, pair_off, grid_off;
    int n_atoms, R, T, n_pairs, max_depth, local_steps, n_grid;
    int lane;
    int lig;
    __device__ __forceinline__ const AtomRec* atoms() const { return B->atoms + atom_off; }
    // the staged copies (make_ctx) in this warp's shared memory
    __device__ __forceinline__ AtomRec atom(const Layout& L, int a) const {
#if UD_STAGE_ATOMS
        const float4 v = reinterpret_cast<const float4*>(s + L.atomrec)[a];
#else
        const float4 v = __ldg(reinterpret_cast<const float4*>(B->atoms + atom_off) + a);
#endif
        AtomRec r;
        r.x = v.x; r.y = v.y; r.z = v.z;
        r.packed = __float_as_int(v.w);
        return r;
    }
    __device__ __forceinline__ int atom_packed(const Layout& L, int a) const {
#if UD_STAGE_ATOMS
        return __float_as_int(s[L.atomrec + 4 * a + 3]);
#else
        return __ldg(&B->atoms[atom_off + a].packed);
#endif
    }
    __device__ __forceinline__ uint32_t grid_word(const Layout& L, int k) const {
#if UD_STAGE_ATOMS
        return __float_as_uint(s[L.gridl + k]);
#else
        return __ldg(B->grid_list + grid_off + k);
#endif
    }
    __device__ __forceinline__ const NodeRec* nodes() const { return B->nodes + node_off; }
    __device__ __forceinline__ const uint32_t* pairs() const { return B->pairs + pair_off; }
    // atom | slot << 8 of the atoms with a grid map
    __device__ __forceinline__ const uint32_t* grid() const { return B->grid_list + grid_off; }
    // AD4: atom charges and per pair slot coefficients
    __device__ __forceinline__ const float* q() const { return B->charges + atom_off; }
    __device__ __forceinline__ const float2* coef() const { return B->pair_coef + pair_off; }
};

// The ligand's context, with its atom records and grid-atom words copied into
// the warp's shared memory (read there by every evaluation).
template <int kW = 32>
__device__ __forceinline__ Ctx make_ctx(const Batch& B, int lig, float* s, const Layout& L) {
    Ctx c;
    const LigDesc* d = B.ligs + lig;
    c.s = s;
    c.B = &B;
    c.atom_off = __ldg(&d->atom_off);
    c.node_off = __ldg(&d->node_off);
    c.pair_off = __ldg(&d->pair_off);
    c.grid_off = __ldg(&d->grid_off);
    c.n_grid = __ldg(&d->n_grid);
    c.n_atoms = __ldg(&d->n_atoms);
    c.R = __ldg(&d->n_nodes);
    c.T = c.R - 1;
    c.n_pairs = __ldg(&d->n_pairs);
    c.max_depth = __ldg(&d->max_depth);
    c.local_steps = __ldg(&d->local_steps);
    c.lane = threadIdx.x & (kW - 1);
    c.lig = lig;
#if UD_STAGE_ATOMS
    const float4* ar = reinterpret_cast<const float4*>(B.atoms + c.atom_off);
    float4* sa = reinterpret_cast<float4*>(s + L.atomrec);
    for (int a = c.lane; a < c.n_atoms; a += kW) sa[a] = __ldg(ar + a);
    uint32_t* sg = reinterpret_cast<uint32_t*>(s + L.gridl);
    for (int k = c.lane; k < c.n_grid; k += kW) sg[k] = __ldg(B.grid_list + c.grid_off + k);
    lanes_sync<kW>();
#endif
    return c;
}

// ---------------------------------------------------------------- evaluation
// Forward kinematics: node frames by tree depth, then atom coordinates.
// A branch's orientation is its parent's composed with the torsion rotation
// about the branch axis; written in the parent's frame that rotation
// (axis_angle(rel_axis, theta)) does not depend on the parent, so all torsion
// quaternions are formed in one parallel pass and each tree level only
// composes q_parent * t (equal to axis_angle(R_parent rel_axis, theta) * q_parent
// of tree.h:116-128 for unit quaternions).
template <int kW = 32>
__device__ __forceinline__ void kinematics(const Ctx& c, const Layout& L, const float* conf) {
    float* fr = c.s + L.frames;
    const NodeRec* nodes = c.nodes();
    // frame layout (20 floats): origin[0..2] q[3..6] R[7..15] lab axis[16..18];
    // [16..19] hold the local torsion quaternion until the node is composed.
    // A lane's first node (1 + lane) is read from global memory once and kept
    // in registers for the torsion pass and every tree level; nodes past the
    // lanes (more than kW - 1 torsions) are read where they are used.
    const int n0 = 1 + c.lane;
    float ro0[3] = {0.0f, 0.0f, 0.0f}, ra0[3] = {0.0f, 0.0f, 0.0f};
    int par0 = 0, dep0 = 0;
    if (n0 < c.R) {
        const NodeRec* nr = nodes + n0;
        ro0[0] = __ldg(&nr->rel_origin[0]); ro0[1] = __ldg(&nr->rel_origin[1]); ro0[2] = __ldg(&nr->rel_origin[2]);
        ra0[0] = __ldg(&nr->rel_axis[0]); ra0[1] = __ldg(&nr->rel_axis[1]); ra0[2] = __ldg(&nr->rel_axis[2]);
        par0 = __ldg(&nr->parent);
        dep0 = __ldg(&nr->depth);
    }
    for (int n = n0; n < c.R; n += kW) {
        float ra[3] = {ra0[0], ra0[1], ra0[2]};
        if (n != n0) {
            const NodeRec* nr = nodes + n;
            ra[0] = __ldg(&nr->rel_axis[0]); ra[1] = __ldg(&nr->rel_axis[1]); ra[2] = __ldg(&nr->rel_axis[2]);
        }
        float tq[4];
        axis_angle_q(ra, conf[7 + n - 1], tq);
        reinterpret_cast<float4*>(fr + 20 * n)[4] = make_float4(tq[0], tq[1], tq[2], tq[3]);
    }
    if (c.lane == 0) {
        fr[0] = conf[0]; fr[1] = conf[1]; fr[2] = conf[2];
        fr[3] = conf[3]; fr[4] = conf[4]; fr[5] = conf[5]; fr[6] = conf[6];
        q_to_r3(fr + 3, fr + 7);
    }
    lanes_sync<kW>();
    for (int d = 1; d <= c.max_depth; ++d) {
        for (int n = n0; n < c.R; n += kW) {
            float ro[3] = {ro0[0], ro0[1], ro0[2]}, ra[3] = {ra0[0], ra0[1], ra0[2]};
            int parent = par0, depth = dep0;
            if (n != n0) {
                const NodeRec* nr = nodes + n;
                depth = __ldg(&nr->depth);
                if (depth != d) continue;
                parent = __ldg(&nr->parent);
                ro[0] = __ldg(&nr->rel_origin[0]); ro[1] = __ldg(&nr->rel_origin[1]); ro[2] = __ldg(&nr->rel_origin[2]);
                ra[0] = __ldg(&nr->rel_axis[0]); ra[1] = __ldg(&nr->rel_axis[1]); ra[2] = __ldg(&nr->rel_axis[2]);
            }
            if (depth != d) continue;
            // frames as five float4: (o, q0) (q1..3, R0) (R1..4) (R5..8) (axis, -)
            const float4* pf = reinterpret_cast<const float4*>(fr + 20 * parent);
            float4* f = reinterpret_cast<float4*>(fr + 20 * n);
            const float4 p0 = pf[0], p1 = pf[1], p2 = pf[2], p3 = pf[3], tq = f[4];
            const float pm[9] = {p1.w, p2.x, p2.y, p2.z, p2.w, p3.x, p3.y, p3.z, p3.w};
            const float po[3] = {p0.x, p0.y, p0.z}, pq[4] = {p0.w, p1.x, p1.y, p1.z};
            const float t[4] = {tq.x, tq.y, tq.z, tq.w};
            float o[3], ax[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                o[i] = po[i] + (pm[3 * i] * ro[0] + pm[3 * i + 1] * ro[1] + pm[3 * i + 2] * ro[2]);
                ax[i] = pm[3 * i] * ra[0] + pm[3 * i + 1] * ra[1] + pm[3 * i + 2] * ra[2];
            }
            float q[4], m[9];
            qmul(pq, t, q);
            qnormalize_approx(q);
            q_to_r3(q, m);
            f[0] = make_float4(o[0], o[1], o[2], q[0]);
            f[1] = make_float4(q[1], q[2], q[3], m[0]);
            f[2] = make_float4(m[1], m[2], m[3], m[4]);
            f[3] = make_float4(m[5], m[6], m[7], m[8]);
            f[4] = make_float4(ax[0], ax[1], ax[2], 0.0f);
        }
        lanes_sync<kW>();
    }
    float4* xyz = reinterpret_cast<float4*>(c.s + L.coords);
    for (int a = c.lane; a < c.n_atoms; a += kW) {
        const AtomRec ar = c.atom(L, a);
        const float4* f = reinterpret_cast<const float4*>(fr + 20 * (ar.packed & 0xFF));
        const float4 f0 = f[0], f1 = f[1], f2 = f[2], f3 = f[3];
        const float fo[3] = {f0.x, f0.y, f0.z};
        const float m[9] = {f1.w, f2.x, f2.y, f2.z, f2.w, f3.x, f3.y, f3.z, f3.w};
        float o[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) o[i] = fo[i] + (m[3 * i] * ar.x + m[3 * i + 1] * ar.y + m[3 * i + 2] * ar.z);
        xyz[a] = make_float4(o[0], o[1], o[2], 0.0f);
    }
    lanes_sync<kW>();
}

// Trilinear map energy, gradient and out-of-box penalty of one atom.
__device__ __forceinline__ float grid_eval(const Maps& M, int slot, const float4 pos, float v,
                                           float& gx, float& gy, float& gz, bool want_deriv) {
    float s[3], miss[3];
    int reg[3], a[3];
    const int dims[3] = {M.nx, M.ny, M.nz};
    const float p[3] = {pos.x, pos.y, pos.z};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float si = (p[i] - M.init[i]) * M.factor[i];
        if (si < 0) {
            miss[i] = -si; reg[i] = -1; a[i] = 0; si = 0;
        } else if (si >= M.dim_m1[i]) {
            miss[i] = si - M.dim_m1[i]; reg[i] = 1; a[i] = dims[i] - 2; si = 1;
        } else {
            miss[i] = 0; reg[i] = 0; a[i] = (int)si; si -= a[i];
        }
        s[i] = si;
    }
    const float penalty = M.slope * (miss[0] * M.factor_inv[0] + miss[1] * M.factor_inv[1] +
                                     miss[2] * M.factor_inv[2]);
    // the 8 corners as 4 x-pairs: a[0] <= nx - 2, so x + 1 is always a grid point
    const float2* g = M.xp + (size_t)slot * M.nx * M.ny * M.nz;
    const int sy = M.nx, sz = M.nx * M.ny;
    const int base = a[0] + sy * a[1] + sz * a[2];
    const float2 c00 = ld_stream2(g + base), c10 = ld_stream2(g + base + sy);
    const float2 c01 = ld_stream2(g + base + sz), c11 = ld_stream2(g + base + sy + sz);
    const float f000 = c00.x, f100 = c00.y, f010 = c10.x, f110 = c10.y;
    const float f001 = c01.x, f101 = c01.y, f011 = c11.x, f111 = c11.y;
    const float x = s[0], y = s[1], z = s[2];
    const float mx = 1 - x, my = 1 - y, mz = 1 - z;
    float f = f000 * mx * my * mz + f100 * x * my * mz + f010 * mx * y * mz + f110 * x * y * mz +
              f001 * mx * my * z + f101 * x * my * z + f011 * mx * y * z + f111 * x * y * z;
    if (want_deriv) {
        float xg = -f000 * my * mz + f100 * my * mz - f010 * y * mz + f110 * y * mz -
                   f001 * my * z + f101 * my * z - f011 * y * z + f111 * y * z;
        float yg = -f000 * mx * mz - f100 * x * mz + f010 * mx * mz + f110 * x * mz -
                   f001 * mx * z - f101 * x * z + f011 * mx * z + f111 * x * z;
        float zg = -f000 * mx * my - f100 * x * my - f010 * mx * y - f110 * x * y +
                   f001 * mx * my + f101 * x * my + f011 * mx * y + f111 * x * y;
        if (f > 0 && v < 0.1f * kMaxFl) {  // curl
            float tmp = (v < kEps) ? 0 : __fdividef(v, v + f);
            f *= tmp;
            float t2 = tmp * tmp;
            xg *= t2; yg *= t2; zg *= t2;
        }
        gx = M.factor[0] * (reg[0] == 0 ? xg : 0.0f) + M.slope * reg[0];
        gy = M.factor[1] * (reg[1] == 0 ? yg : 0.0f) + M.slope * reg[1];
        gz = M.factor[2] * (reg[2] == 0 ? zg : 0.0f) + M.slope * reg[2];
    } else {
        if (f > 0 && v < 0.1f * kMaxFl) {
            float tmp = (v < kEps) ? 0 : __fdividef(v, v + f);
            f *= tmp;
        }
    }
    return f + penalty;
}

// The bias wells a ligand is scored with against the receptor atoms: its own
// list when it has one (model::bias_list), else the maps' (non_cache::bias_list).
__device__ __forceinline__ void bias_of(const Receptor& R, int lig, const BiasRec*& bias, int& n) {
    const int span = R.lig_bias_span ? __ldg(R.lig_bias_span + lig) : 0;
    if (span >> 16) {
        bias = R.lig_bias + (span & 0xFFFF);
        n = span >> 16;
    } else {
        bias = R.bias;
        n = R.n_bias;
    }
}

// Interaction of one ligand atom (XS type t1, position pa) with the receptor
// atoms, all lanes of the warp together (non_cache::eval_deriv / eval,
// non_cache.cpp:35-110, 420-500): the position is clamped into the box at a
// penalty of slope x the distance moved (derivative +-slope per axis), the
// pair terms of the receptor atoms within the cutoff of the clamped position
// are summed (lerped (e, dE/dr / r) table rows with kDeriv, the nearest-bin
// `fast` table without), and the sum is curled at cap v.  Every lane returns
// the same energy and gradient.
template <bool kDeriv>
__device__ __forceinline__ float receptor_term(const Receptor& R, const Tables& Tb, int t1, const float4 pa, float v,
                                               float slope, const BiasRec* bias, int n_bias, float& gx, float& gy,
                                               float& gz) {
    const int lane = threadIdx.x & 31;
    float p[3] = {pa.x, pa.y, pa.z};
    float pen = 0, od[3] = {0, 0, 0};
    int ci[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (p[i] < R.begin[i]) {
            pen += R.begin[i] - p[i];
            p[i] = R.begin[i];
            od[i] = -1;
        } else if (p[i] > R.end[i]) {
            pen += p[i] - R.end[i];
            p[i] = R.end[i];
            od[i] = 1;
        }
        int k = (int)((p[i] - R.begin[i]) * R.inv_cell);
        ci[i] = k < 0 ? 0 : (k >= R.n[i] ? R.n[i] - 1 : k);
    }
    const int cell = (ci[2] * R.n[1] + ci[1]) * R.n[0] + ci[0];
    const int j0 = __ldg(R.start + cell), j1 = __ldg(R.start + cell + 1);
    float e = 0, dx = 0, dy = 0, dz = 0;
    for (int j = j0 + lane; j < j1; j += 32) {
        const float4 r = __ldg(R.atoms + j);
        const float rx = p[0] - r.x, ry = p[1] - r.y, rz = p[2] - r.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        if (r2 < Tb.cutoff2) {
            const int t2 = __float_as_int(r.w);
            const int tp = t1 <= t2 ? t1 + t2 * (t2 + 1) / 2 : t2 + t1 * (t1 + 1) / 2;
            const float rf = Tb.factor * r2;
            const int i1 = (int)rf;
            if constexpr (kDeriv) {
                const float4 t = __ldg(Tb.smooth4 + (size_t)tp * Tb.n_bins + i1);
                const float rem = rf - i1;
                e += t.x + rem * (t.z - t.x);
                const float dor = t.y + rem * (t.w - t.y);
                dx += dor * rx;
                dy += dor * ry;
                dz += dor * rz;
            } else {
                e += __ldg(Tb.fast + (size_t)tp * Tb.n_bins + i1);
            }
        }
    }
    e = warp_sum(e);
    if constexpr (kDeriv) {
        dx = warp_sum(dx);
        dy = warp_sum(dy);
        dz = warp_sum(dz);
    }
    if (n_bias > 0) {  // bias wells at the unclamped position, before the curl (non_cache.cpp:112-400)
        for (int k = 0; k < n_bias; ++k) {
            const BiasRec* b = bias + k;
            const int m = __ldg(&b->mult[t1]);
            if (m == 0) continue;
            const float bx = pa.x - __ldg(&b->x), by = pa.y - __ldg(&b->y), bz = pa.z - __ldg(&b->z);
            const float rb2 = bx * bx + by * by + bz * bz;
            if (rb2 > Tb.cutoff2) continue;
            const float r = __ldg(&b->r);
            const float dE = __ldg(&b->vset) * expf(-rb2 / r / r);
            if (dE >= -0.01f) continue;
            const float f = dE / (-r * r);
            for (int q = 0; q < m; ++q) {
                e += dE;
                if constexpr (kDeriv) {
                    dx += f * bx;
                    dy += f * by;
                    dz += f * bz;
                }
            }
        }
    }
    if (e > 0 && v < 0.1f * kMaxFl) {  // curl
        const float tmp = (v < kEps) ? 0 : v / (v + e);
        e *= tmp;
        const float t2 = tmp * tmp;
        dx *= t2; dy *= t2; dz *= t2;
    }
    gx = dx + od[0] * slope;
    gy = dy + od[1] * slope;
    gz = dz + od[2] * slope;
    return e + pen * slope;
}

// Energy and gradient (change layout: position, torque, torsions) of `conf`.
// Pair forces use the table's dE/dr / r column (precalculate.h:48-65) or, with
// kExactPairs, the slope of the lerped energy itself.
// With kReceptor the receptor term comes from the receptor atoms (`Rc`,
// out-of-box slope `rslope`) instead of the maps.
template <bool kExactPairs = false, bool kAD4 = false, bool kReceptor = false, int kW = 32>
__device__ __forceinline__ float eval_deriv(const Ctx& c, const Layout& L, const Maps& M,
                                            const Tables& Tb, const float* conf, float* g,
                                            float v_intra, float v_inter, const Receptor* Rc = nullptr,
                                            float rslope = 0.0f) {
    static_assert(!kReceptor || kW == 32, "receptor-atom terms use the whole warp");
    kinematics<kW>(c, L, conf);
    const float4* xyz = reinterpret_cast<const float4*>(c.s + L.coords);
    float4* frc = reinterpret_cast<float4*>(c.s + L.forces);
    // pair forces of the odd lane ranges (UD_FORCE_SPLIT), summed into the
    // per-atom forces by the prefix scan
    float4* frc2 = reinterpret_cast<float4*>(c.s + L.forces2);
    float e = 0;
    // the per-atom force array: the grid (or receptor-atom) force of every
    // atom, then the pair forces
    for (int k = c.lane; k < c.n_atoms; k += kW) {
        frc[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (UD_FORCE_SPLIT == 2) frc2[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    lanes_sync<kW>();
    if constexpr (kReceptor) {
        const BiasRec* bias;
        int n_bias;
        bias_of(*Rc, c.lig, bias, n_bias);
        for (int k = 0; k < c.n_grid; ++k) {  // one atom at a time, lanes over its receptor atoms
            const int a = c.grid_word(L, k) & 0xFF;
            const int t1 = ((c.atom_packed(L, a) >> 24) & 0xFF) - 1;
            float gx, gy, gz;
            const float ea = receptor_term<true>(*Rc, Tb, t1, xyz[a], v_inter, rslope, bias, n_bias, gx, gy, gz);
            if (c.lane == 0) {
                frc[a] = make_float4(gx, gy, gz, 0.0f);
                e += ea;
            }
        }
    } else {
        // grid energy and gradient (grid.cpp:40-129) over the compacted list of
        // atoms with a map: one pass of lanes, so that all corner loads of a
        // ligand of up to kW heavy atoms are in flight together
        for (int k = c.lane; k < c.n_grid; k += kW) {
            const uint32_t ga = c.grid_word(L, k);
            const int a = ga & 0xFF, slot = ga >> 8;
            float gx, gy, gz;
            const float4 pa = xyz[a];
            e += grid_eval(M, slot, pa, v_inter, gx, gy, gz, true);
            if constexpr (kAD4) {  // electrostatic map x q, desolvation map x |q| (ad4cache.cpp:227-269)
                const float q = __ldg(c.q() + a), aq = fabsf(q);
                float hx, hy, hz;
                e += q * grid_eval(M, M.e_slot, pa, v_inter, hx, hy, hz, true);
                gx += q * hx; gy += q * hy; gz += q * hz;
                e += aq * grid_eval(M, M.d_slot, pa, v_inter, hx, hy, hz, true);
                gx += aq * hx; gy += aq * hy; gz += aq * hz;
            }
            frc[a] = make_float4(gx, gy, gz, 0.0f);
        }
    }
    lanes_sync<kW>();
    // Pairs in 32-slot groups made of kPairPasses lane ranges that are each a
    // matching (no atom twice within a range), taken kW slots (a window of
    // whole ranges) at a time; the ranges add their forces in a fixed order
    // of passes (no atomics, a fixed summation order).  The software-pipelined
    // loop (UD_PAIR_PIPE) runs by default; the loop after it loads the table
    // rows of kPairBatch windows before consuming any.
    static_assert(kW % kPairPassWidth == 0, "a window holds whole lane ranges");
    constexpr int kWinShift = kW == 32 ? 5 : 4;
    constexpr int kWinPasses = kW / kPairPassWidth;
    const int n_groups = c.n_pairs >> kWinShift;   // windows; n_pairs is a multiple of 32
    // with UD_PAIR_PREFETCH the next window's pair word is loaded while this
    // window is worked on, so its latency is off the window's dependent chain
    uint32_t pr_next = (UD_PAIR_PREFETCH && n_groups > 0) ? __ldg(c.pairs() + c.lane) : kPairPad;
#if UD_PAIR_PIPE
    // Software-pipelined windows: the table row (AD4: and the E and G rows) of window
    // g + UD_PAIR_PIPE is requested before window g's forces are added (and
    // its pair word one window earlier), so each window's L2 round trip
    // overlaps the work of the windows before it.
    if constexpr (!kAD4 || UD_PAIR_PIPE_AD4) {
        constexpr int kPipe = UD_PAIR_PIPE;
        constexpr int kSplit = UD_FORCE_SPLIT;
        const int range = c.lane / kPairPassWidth;
        float4* fd = (kSplit == 2 && (range & 1)) ? frc2 : frc;
        const uint32_t* pw = c.pairs() + c.lane;
        struct Stage {
            uint32_t pr;   // pair word, kPairPad when the slot adds nothing
            float4 t;      // table row (e_i, dor_i, e_i+1, dor_i+1)
            float rem, rx, ry, rz;
            float4 te, tg; // AD4: the shared E and G rows and the pair's scales of them
            float2 cf;
        };
        auto request = [&](int g, uint32_t w, Stage& q) {
            q.pr = kPairPad;
            q.t = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            q.rem = q.rx = q.ry = q.rz = 0.0f;
            if constexpr (kAD4) {
                q.te = q.tg = q.t;
                q.cf = make_float2(0.0f, 0.0f);
            }
            if (w != kPairPad) {
                const float4 pa = xyz[w & 0xFF], pb = xyz[(w >> 8) & 0xFF];
                q.rx = pb.x - pa.x; q.ry = pb.y - pa.y; q.rz = pb.z - pa.z;
                const float r2 = q.rx * q.rx + q.ry * q.ry + q.rz * q.rz;
                if (r2 < Tb.cutoff2) {
                    const float rf = Tb.factor * r2;
                    const int i1 = (int)rf;
                    q.rem = rf - i1;
                    q.t = ld_stream4(Tb.smooth4 + (size_t)(w >> 16) * Tb.n_bins + i1);
                    if constexpr (kAD4) {  // + q_a q_b E(r) + (|q_a| V_b + |q_b| V_a) G(r)
                        q.cf = __ldg(c.coef() + (g << kWinShift) + c.lane);
                        q.te = __ldg(Tb.smooth4 + (size_t)kAd4RowE * Tb.n_bins + i1);
                        q.tg = __ldg(Tb.smooth4 + (size_t)kAd4RowG * Tb.n_bins + i1);
                    }
                    q.pr = w;
                }
            }
        };
        auto word = [&](int g) { return g < n_groups ? __ldg(pw + (g << kWinShift)) : kPairPad; };
        Stage q[kPipe + 1];
#pragma unroll
        for (int k = 0; k < kPipe; ++k) request(k, word(k), q[k]);
        uint32_t w_next = word(kPipe);
        for (int g = 0; g < n_groups; ++g) {
            const uint32_t w1 = w_next;
            w_next = word(g + kPipe + 1);
            request(g + kPipe, w1, q[kPipe]);
            const Stage& h = q[0];
            float fx = 0, fy = 0, fz = 0;
            const bool live = h.pr != kPairPad;
            if (live) {
                float4 t = h.t;
                if constexpr (kAD4) {
                    t.x += h.cf.x * h.te.x + h.cf.y * h.tg.x;
                    t.y += h.cf.x * h.te.y + h.cf.y * h.tg.y;
                    t.z += h.cf.x * h.te.z + h.cf.y * h.tg.z;
                    t.w += h.cf.x * h.te.w + h.cf.y * h.tg.w;
                }
                float ep = t.x + h.rem * (t.z - t.x);
                float dor = kExactPairs ? 2.0f * Tb.factor * (t.z - t.x) : t.y + h.rem * (t.w - t.y);
                fx = dor * h.rx; fy = dor * h.ry; fz = dor * h.rz;
                if (ep > 0 && v_intra < 0.1f * kMaxFl) {
                    float tmp = (v_intra < kEps) ? 0 : __fdividef(v_intra, v_intra + ep);
                    ep *= tmp;
                    float t2 = tmp * tmp;
                    fx *= t2; fy *= t2; fz *= t2;
                }
                e += ep;
            }
            const int a = h.pr & 0xFF, b = (h.pr >> 8) & 0xFF;
#pragma unroll
            for (int pass = 0; pass < kWinPasses / kSplit; ++pass) {
                if (live && range / kSplit == pass) {
                    float4 fa = fd[a], fb = fd[b];
                    fa.x -= fx; fa.y -= fy; fa.z -= fz;
                    fb.x += fx; fb.y += fy; fb.z += fz;
                    fd[a] = fa;
                    fd[b] = fb;
                }
                lanes_sync<kW>();
            }
#pragma unroll
            for (int k = 0; k < kPipe; ++k) q[k] = q[k + 1];
        }
    } else
#endif
    for (int g0 = 0; g0 < n_groups; g0 += kPairBatch) {
        float4 tv[kPairBatch];
        float rv[kPairBatch][3];
        float remv[kPairBatch];
        uint32_t prv[kPairBatch];
#pragma unroll
        for (int u = 0; u < kPairBatch; ++u) {
            prv[u] = kPairPad;
            if (g0 + u < n_groups) {
                uint32_t pr;
                if (UD_PAIR_PREFETCH && kPairBatch == 1) {
                    pr = pr_next;
                    pr_next = g0 + 1 < n_groups ? __ldg(c.pairs() + ((g0 + 1) << kWinShift) + c.lane) : kPairPad;
                } else {
                    pr = __ldg(c.pairs() + ((g0 + u) << kWinShift) + c.lane);
                }
                if (pr != kPairPad) {
                    int a = pr & 0xFF, b = (pr >> 8) & 0xFF, tp = pr >> 16;
                    const float4 pa = xyz[a], pb = xyz[b];
                    float rx = pb.x - pa.x, ry = pb.y - pa.y, rz = pb.z - pa.z;
                    float r2 = rx * rx + ry * ry + rz * rz;
                    if (r2 < Tb.cutoff2) {
                        float rf = Tb.factor * r2;
                        int i1 = (int)rf;
                        remv[u] = rf - i1;
                        rv[u][0] = rx; rv[u][1] = ry; rv[u][2] = rz;
                        tv[u] = ld_stream4(Tb.smooth4 + (size_t)tp * Tb.n_bins + i1);
                        if constexpr (kAD4) {  // + q_a q_b E(r) + (|q_a| V_b + |q_b| V_a) G(r)
                            const float2 cf = __ldg(c.coef() + ((g0 + u) << kWinShift) + c.lane);
                            const float4 te = __ldg(Tb.smooth4 + (size_t)kAd4RowE * Tb.n_bins + i1);
                            const float4 tg = __ldg(Tb.smooth4 + (size_t)kAd4RowG * Tb.n_bins + i1);
                            tv[u].x += cf.x * te.x + cf.y * tg.x;
                            tv[u].y += cf.x * te.y + cf.y * tg.y;
                            tv[u].z += cf.x * te.z + cf.y * tg.z;
                            tv[u].w += cf.x * te.w + cf.y * tg.w;
                        }
                        prv[u] = pr;
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kPairBatch; ++u) {
            float fx = 0, fy = 0, fz = 0;
            const bool live = prv[u] != kPairPad;
            if (live) {
                const float4 t = tv[u];
                const float rem = remv[u];
                float ep = t.x + rem * (t.z - t.x);
                float dor = kExactPairs ? 2.0f * Tb.factor * (t.z - t.x) : t.y + rem * (t.w - t.y);
                fx = dor * rv[u][0]; fy = dor * rv[u][1]; fz = dor * rv[u][2];
                if (ep > 0 && v_intra < 0.1f * kMaxFl) {
                    float tmp = (v_intra < kEps) ? 0 : __fdividef(v_intra, v_intra + ep);
                    ep *= tmp;
                    float t2 = tmp * tmp;
                    fx *= t2; fy *= t2; fz *= t2;
                }
                e += ep;
            }
            const int a = prv[u] & 0xFF, b = (prv[u] >> 8) & 0xFF;
            // ranges 2p and 2p + 1 add in pass p, one into each force array
            // (a range is a matching, so no atom is written twice in a pass)
            constexpr int kSplit = UD_FORCE_SPLIT;
            const int range = c.lane / kPairPassWidth;
            float4* fd = (kSplit == 2 && (range & 1)) ? frc2 : frc;
#pragma unroll
            for (int pass = 0; pass < kWinPasses / kSplit; ++pass) {
                if (live && range / kSplit == pass) {
                    float4 fa = fd[a], fb = fd[b];
                    fa.x -= fx; fa.y -= fy; fa.z -= fz;
                    fb.x += fx; fb.y += fy; fb.z += fz;
                    fd[a] = fa;
                    fd[b] = fb;
                }
                lanes_sync<kW>();
            }
        }
    }
    e = lanes_sum<kW>(e);
    // Force and torque of every subtree.  A subtree's atoms are contiguous in
    // DFS order, so inclusive prefix sums over atoms of f and of the moment
    // (x - o_root) x f give each subtree's sums as a difference of two
    // prefixes; the torque about the subtree's own origin o is then
    // M - (o - o_root) x F (tree.h:75-84,164-192 sum the same terms node by node).
    const float* fr = c.s + L.frames;
    float* pre = c.s + L.prefix;
    float carry[6] = {0, 0, 0, 0, 0, 0};
    const unsigned lanes = lanes_mask<kW>();
    for (int base = 0; base < c.n_atoms; base += kW) {
        const int a = base + c.lane;
        float v[6] = {0, 0, 0, 0, 0, 0};
        if (a < c.n_atoms) {
            float4 fa = frc[a];
            if (UD_FORCE_SPLIT == 2) {
                const float4 fb = frc2[a];
                fa.x += fb.x; fa.y += fb.y; fa.z += fb.z;
            }
            const float4 xa = xyz[a];
            const float f0 = fa.x, f1 = fa.y, f2 = fa.z;
            const float r0 = xa.x - fr[0], r1 = xa.y - fr[1], r2 = xa.z - fr[2];
            v[0] = f0; v[1] = f1; v[2] = f2;
            v[3] = r1 * f2 - r2 * f1;
            v[4] = r2 * f0 - r0 * f2;
            v[5] = r0 * f1 - r1 * f0;
        }
#pragma unroll
        for (int off = 1; off < kW; off <<= 1) {
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const float t = __shfl_up_sync(lanes, v[q], off, kW);
                if (c.lane >= off) v[q] += t;
            }
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            v[q] += carry[q];
            carry[q] = __shfl_sync(lanes, v[q], kW - 1, kW);
        }
        if (a < c.n_atoms) {  // 6 floats an atom: three 8-byte stores
            float2* pa = reinterpret_cast<float2*>(pre + 6 * a);
            pa[0] = make_float2(v[0], v[1]);
            pa[1] = make_float2(v[2], v[3]);
            pa[2] = make_float2(v[4], v[5]);
        }
    }
    lanes_sync<kW>();
    for (int n = c.lane; n < c.R; n += kW) {
        const int span = __ldg(&c.nodes()[n].atoms);
        const int b0 = span & 0xFFFF, b1 = span >> 16;
        const float2* hi = reinterpret_cast<const float2*>(pre + 6 * (b1 - 1));
        const float2 h0 = hi[0], h1 = hi[1], h2 = hi[2];
        float2 l0 = make_float2(0.0f, 0.0f), l1 = l0, l2 = l0;
        if (b0 > 0) {
            const float2* lo = reinterpret_cast<const float2*>(pre + 6 * (b0 - 1));
            l0 = lo[0]; l1 = lo[1]; l2 = lo[2];
        }
        const float sm[6] = {h0.x - l0.x, h0.y - l0.y, h1.x - l1.x, h1.y - l1.y, h2.x - l2.x, h2.y - l2.y};
        const float* on = fr + 20 * n;
        const float d0 = on[0] - fr[0], d1 = on[1] - fr[1], d2 = on[2] - fr[2];
        const float T0 = sm[3] - (d1 * sm[2] - d2 * sm[1]);
        const float T1 = sm[4] - (d2 * sm[0] - d0 * sm[2]);
        const float T2 = sm[5] - (d0 * sm[1] - d1 * sm[0]);
        if (n == 0) {
            g[0] = sm[0]; g[1] = sm[1]; g[2] = sm[2];
            g[3] = T0; g[4] = T1; g[5] = T2;
        } else {
            g[6 + n - 1] = T0 * on[16] + T1 * on[17] + T2 * on[18];
        }
    }
    lanes_sync<kW>();
    return e;
}

// Intramolecular energy from the nearest-bin `fast` table at curl cap v
// (model::evali, model.cpp:927-933), summed over the warp.
template <bool kAD4 = false, int kW = 32>
__device__ __forceinline__ float intra_fast(const Ctx& c, const Tables& Tb, const float4* xyz, float v) {
    float ei = 0;
    for (int k = c.lane; k < c.n_pairs; k += kW) {
        uint32_t pr = __ldg(c.pairs() + k);
        if (pr == kPairPad) continue;
        int a = pr & 0xFF, b = (pr >> 8) & 0xFF, tp = pr >> 16;
        const float4 pa = xyz[a], pb = xyz[b];
        float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
        float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < Tb.cutoff2) {
            const int bin = (int)(Tb.factor * r2);
            float t = __ldg(Tb.fast + (size_t)tp * Tb.n_bins + bin);
            if constexpr (kAD4) {
                const float2 cf = __ldg(c.coef() + k);
                t += cf.x * __ldg(Tb.fast + (size_t)kAd4RowE * Tb.n_bins + bin) +
                     cf.y * __ldg(Tb.fast + (size_t)kAd4RowG * Tb.n_bins + bin);
            }
            if (t > 0 && v < 0.1f * kMaxFl) t *= (v < kEps) ? 0 : __fdividef(v, v + t);
            ei += t;
        }
    }
    return lanes_sum<kW>(ei);
}

// Scoring-path energy (no gradient): grid with curl cap v, intramolecular
// pairs from the nearest-bin `fast` table (model.cpp:867-886, cache.cpp:84-120).
template <bool kAD4 = false, int kW = 32>
__device__ __forceinline__ void eval_score(const Ctx& c, const Layout& L, const Maps& M,
                                           const Tables& Tb, const float* conf, float v,
                                           float& e_grid, float& e_intra) {
    kinematics<kW>(c, L, conf);
    const float4* xyz = reinterpret_cast<const float4*>(c.s + L.coords);
    float eg = 0;
    for (int k = c.lane; k < c.n_grid; k += kW) {
        const uint32_t ga = c.grid_word(L, k);
        float gx, gy, gz;
        const float4 pa = xyz[ga & 0xFF];
        eg += grid_eval(M, ga >> 8, pa, v, gx, gy, gz, false);
        if constexpr (kAD4) {
            const float q = __ldg(c.q() + (ga & 0xFF));
            eg += q * grid_eval(M, M.e_slot, pa, v, gx, gy, gz, false);
            eg += fabsf(q) * grid_eval(M, M.d_slot, pa, v, gx, gy, gz, false);
        }
    }
    e_grid = lanes_sum<kW>(eg);
    e_intra = intra_fast<kAD4, kW>(c, Tb, xyz, v);
}

// ---------------------------------------------------------------- BFGS pieces
template <int kW = 32>
__device__ __forceinline__ float dotw(const Ctx& c, const float* a, const float* b, int n) {
    float s = 0;
    for (int i = c.lane; i < n; i += kW) s += a[i] * b[i];
    return lanes_sum<kW>(s);
}

template <int kW = 32>
__device__ __forceinline__ void copyw(const Ctx& c, float* dst, const float* src, int n) {
    for (int i = c.lane; i < n; i += kW) dst[i] = src[i];
    lanes_sync<kW>();
}

// x_new = x + alpha * p in conformation space (conf.h:98-104, 146-150).
template <int kW = 32>
__device__ __forceinline__ void conf_increment(const Ctx& c, const float* x, const float* p,
                                               float alpha, float* out) {
    if (c.lane < 3) out[c.lane] = x[c.lane] + alpha * p[c.lane];
    if (c.lane == 3) {
        float rot[3] = {alpha * p[3], alpha * p[4], alpha * p[5]};
        float q[4] = {x[3], x[4], x[5], x[6]};
        quaternion_increment(q, rot);
        out[3] = q[0]; out[4] = q[1]; out[5] = q[2]; out[6] = q[3];
    }
    for (int t = c.lane; t < c.T; t += kW) {
        float v = x[7 + t] + normalized_angle(alpha * p[6 + t]);
        out[7 + t] = normalized_angle(v);
    }
    lanes_sync<kW>();
}

// The inverse Hessian is kept as a full symmetric n x n matrix (the reference
// stores the upper triangle, bfgs.h:27-58): lane i owns row/column i, so both
// products and the update are one contiguous loop per lane.  (Two lanes per
// row for n <= 16 measured no faster: the combining shuffle costs what the
// shorter loops save.)
// out = -H v
template <int kW = 32>
__device__ __forceinline__ void minus_hv(const Ctx& c, const float* H, const float* v, float* out, int n) {
    for (int i = c.lane; i < n; i += kW) {
        float sum = 0;
        for (int j = 0; j < n; ++j) sum += H[j * n + i] * v[j];
        out[i] = -sum;
    }
    lanes_sync<kW>();
}

// out = -H v as minus_hv, returning the dot product out . w, summed as dotw
// does (the lane's terms in order of i, then the shuffle tree).
template <int kW = 32>
__device__ __forceinline__ float minus_hv_dot(const Ctx& c, const float* H, const float* v, float* out,
                                              const float* w, int n) {
    float d = 0;
    for (int i = c.lane; i < n; i += kW) {
        float sum = 0;
        for (int j = 0; j < n; ++j) sum += H[j * n + i] * v[j];
        out[i] = -sum;
        d += -sum * w[i];
    }
    lanes_sync<kW>();
    return lanes_sum<kW>(d);
}

template <int kW = 32>
__device__ __forceinline__ void h_identity(const Ctx& c, float* H, int n) {
    for (int k = c.lane; k < n * n; k += kW) H[k] = 0;
    lanes_sync<kW>();
    for (int i = c.lane; i < n; i += kW) H[i * n + i] = 1;
    lanes_sync<kW>();
}

// BFGS update of the inverse Hessian (bfgs.h:40-58), applied to both triangles
template <int kW = 32>
__device__ __forceinline__ void h_update(const Ctx& c, float* H, const float* p, const float* y,
                                         float* mhy, float alpha, int n, float yp) {
    if (alpha * yp < kEps) return;
    const float yhy = -minus_hv_dot<kW>(c, H, y, mhy, y, n);
    const float r = __frcp_rn(alpha * yp);
    const float a1 = alpha * r, a2 = alpha * alpha * (r * r * yhy + r);
    for (int i = c.lane; i < n; i += kW) {
        const float mi = mhy[i], pi = p[i];
        for (int j = 0; j < n; ++j) H[j * n + i] += a1 * (mi * p[j] + mhy[j] * pi) + a2 * pi * p[j];
    }
    lanes_sync<kW>();
}

// ---------------------------------------------------------------- MC pieces
__device__ void random_inside_sphere(Philox& rng, float* v) {
    for (int it = 0; it < 64; ++it) {
        uint4 u = rng.next();
        float a = 2 * u01(u.x) - 1, b = 2 * u01(u.y) - 1, d = 2 * u01(u.z) - 1;
        float r2 = a * a + b * b + d * d;
        if (r2 < 1 && sqrtf(r2) > 10 * kEps) {
            v[0] = a; v[1] = b; v[2] = d;
            return;
        }
    }
    v[0] = v[1] = v[2] = 0;
}

// Initial chain conformation: position uniform in the box, orientation a
// normalised 4-D Gaussian, torsions uniform (conf.h:105-108,173-176; quaternion.cpp:116-126).
template <int kW = 32>
__device__ void random_conf(const Ctx& c, Philox& rng, const Maps& M, float* x) {
    if (c.lane == 0) {
        uint4 u = rng.next();
        x[0] = M.init[0] + (M.corner2[0] - M.init[0]) * u01(u.x);
        x[1] = M.init[1] + (M.corner2[1] - M.init[1]) * u01(u.y);
        x[2] = M.init[2] + (M.corner2[2] - M.init[2]) * u01(u.z);
        x[3] = 1; x[4] = x[5] = x[6] = 0;
        for (int it = 0; it < 16; ++it) {
            uint4 a = rng.next();
            // Box-Muller with angles in [-pi, pi): sin/cos from the half angle
            float r1 = sqrtf(-2.0f * __logf(fmaxf(u01(a.x), 1e-12f)));
            float r2 = sqrtf(-2.0f * __logf(fmaxf(u01(a.z), 1e-12f)));
            float s1, c1, s2, c2;
            sincos_half(0.5f * (2 * kPi * u01(a.y) - kPi), &s1, &c1);
            sincos_half(0.5f * (2 * kPi * u01(a.w) - kPi), &s2, &c2);
            float q[4] = {r1 * (c1 * c1 - s1 * s1), r1 * (2 * s1 * c1), r2 * (c2 * c2 - s2 * s2),
                          r2 * (2 * s2 * c2)};
            float nrm = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
            if (nrm > kEps) {
                x[3] = q[0] / nrm; x[4] = q[1] / nrm; x[5] = q[2] / nrm; x[6] = q[3] / nrm;
                break;
            }
        }
        for (int t = 0; t < c.T; t += 4) {
            uint4 a = rng.next();
            uint32_t w[4] = {a.x, a.y, a.z, a.w};
            for (int k = 0; k < 4 && t + k < c.T; ++k) x[7 + t + k] = -kPi + 2 * kPi * u01(w[k]);
        }
    }
    lanes_sync<kW>();
}

// Mutation of one of {position, orientation, one torsion} (mutate.cpp:36-80);
// the gyration radius uses the coordinates of the last evaluation.
template <int kW = 32>
__device__ void mutate(const Ctx& c, const Layout& L, Philox& rng, float amplitude, float* x) {
    float* misc = c.s + L.misc;
    if (c.lane == 0) {
        uint4 u = rng.next();
        int which = (int)(u.x % (uint32_t)(2 + c.T));
        float sph[3];
        random_inside_sphere(rng, sph);
        misc[0] = __int_as_float(which);
        misc[1] = sph[0]; misc[2] = sph[1]; misc[3] = sph[2];
        misc[4] = -kPi + 2 * kPi * u01(u.y);
    }
    lanes_sync<kW>();
    const int which = __float_as_int(misc[0]);
    if (which == 1) {
        // gyration radius of heavy atoms about the root origin (model.cpp:853-865)
        const float4* xyz = reinterpret_cast<const float4*>(c.s + L.coords);
        const float* o = c.s + L.frames;
        float acc = 0, cnt = 0;
        for (int a = c.lane; a < c.n_atoms; a += kW) {
            int packed = c.atom_packed(L, a);
            if ((packed >> 16) & 1) {
                const float4 pa = xyz[a];
                float dx = pa.x - o[0], dy = pa.y - o[1], dz = pa.z - o[2];
                acc += dx * dx + dy * dy + dz * dz;
                cnt += 1;
            }
        }
        acc = lanes_sum<kW>(acc);
        cnt = lanes_sum<kW>(cnt);
        float gr = cnt > 0 ? sqrtf(acc / cnt) : 0;
        if (c.lane == 0 && gr > kEps) {
            float rot[3] = {amplitude / gr * misc[1], amplitude / gr * misc[2], amplitude / gr * misc[3]};
            float q[4] = {x[3], x[4], x[5], x[6]};
            quaternion_increment(q, rot);
            x[3] = q[0]; x[4] = q[1]; x[5] = q[2]; x[6] = q[3];
        }
    } else if (c.lane == 0) {
        if (which == 0) {
            x[0] += amplitude * misc[1];
            x[1] += amplitude * misc[2];
            x[2] += amplitude * misc[3];
        } else {
            x[7 + which - 2] = misc[4];
        }
    }
    lanes_sync<kW>();
}

// ---------------------------------------------------------------- chain driver
// States of the per-warp machine.  Everything between two evaluations is
// warp-uniform control; each pass through the loop performs exactly one
// evaluation (eval_x, eval_g) unless the chain or the work runs out.
enum : int {
    S_FETCH = 0,     // take the next (ligand, chain) item
    S_MC_STEP,       // mutate and start the search BFGS, or finish the chain
    S_BFGS_BEGIN,    // identity inverse Hessian, evaluate the start point
    S_BFGS_INIT,     // consume the start-point evaluation
    S_BFGS_ITER,     // new search direction, first line-search trial
    S_LS_DONE,       // consume a line-search evaluation
    S_BFGS_END,      // restore if no improvement, hand the energy back
    S_AFTER_SEARCH,  // Metropolis test of a locally optimised candidate
    S_AFTER_REFINE,  // record the refined pose
    S_DONE,          // write the chain's result
    S_EXIT
};

struct Machine {
    // chain
    int item, lig, chain, step, evals, steps_cap;
    float tmp_e, best_e;
    // BFGS
    int mode;          // 0 candidate search, 1 refinement, 2 standalone optimisation
    int bx_off;        // shared-memory offset of the conformation being optimised
    float v;
    int iter, trial;
    float alpha, f0, f_orig, pg, last_e;
};

// Nanoseconds of the GPU's global timer.
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Loads of stream control words, which host copies write while the kernel
// runs: volatile asm (never merged with an earlier load or hoisted out of a
// wait loop) at GPU scope (read where the copies land, not from a line cached
// in L1).  The acquire load of the published count orders the reads of the
// slot's data after it.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The next (ligand, chain) item of a streaming screen for lane 0 of a chain
// (StreamView): the item's global ligand id and chain, or -1 when the stream
// is closed and drained, the arena is exhausted, or a wait for a publication
// ran past the time limit (status set to kStreamTimeout).
__device__ __noinline__ int stream_fetch(const StreamView& SV, int E, int* item_out, int* chain_out) {
    const unsigned per_slot = (unsigned)SV.slot_ligands * (unsigned)E;
    for (;;) {
        const unsigned it = atomicAdd(SV.next_item, 1u);
        const unsigned s = it / per_slot;
        if (s >= (unsigned)SV.max_slots) return -1;
        unsigned pub = ld_acquire_u32(SV.published);
        if (pub <= s) {
            // the limit runs from the last publication seen: a slot far ahead
            // waits as long as the host keeps publishing earlier ones
            unsigned long long t0 = global_ns();
            for (;;) {
                const unsigned now = ld_acquire_u32(SV.published);
                if (now > s) break;
                if (now != pub) {
                    pub = now;
                    t0 = global_ns();
                }
                if (ld_acquire_u32(SV.closed)) {
                    if (ld_acquire_u32(SV.published) > s) break;
                    return -1;
                }
                if (global_ns() - t0 > SV.timeout_ns) {
                    atomicExch(SV.status, kStreamTimeout);
                    return -1;
                }
                __nanosleep(2000);
            }
        }
        const unsigned within = it - s * per_slot;
        const int l = (int)(within / (unsigned)E);
        if (l >= ld_relaxed_s32(SV.slot_nlig + s)) continue;  // past the slot's ligands
        *item_out = (int)it;
        *chain_out = (int)(within % (unsigned)E);
        return ld_relaxed_s32(SV.order + (size_t)s * SV.slot_ligands + l);
    }
}

// The MC chain of monte_carlo.cu:237-356 (mutate, BFGS at the hunt cap,
// Metropolis at temperature T, refine improvements at the authentic cap, keep
// the best) with the line search and BFGS iterations of bfgs.h:63-146.
template <bool kSearch, bool kAD4, int kW, bool kStream = false>
__device__ __forceinline__ void run_machine(const Batch& B, const Maps& M, const Tables& Tb,
                                            const SearchParams& P, const Layout& L, float* sw,
                                            const int* order, int n_items, int first_item,
                                            unsigned int* queue, float* poses, int pose_stride,
                                            ChainResult* results, const int* opt_lig, int opt_steps,
                                            float opt_v, float* opt_e, int* opt_evals,
                                            const StreamView* SV = nullptr) {
    const int lane = threadIdx.x & (kW - 1);
    const int slot_in_block = threadIdx.x / kW;    // this chain's index in the CTA
    const int chains_in_block = blockDim.x / kW;
    Machine m;
    Ctx c;
    Philox rng;
    int st = S_FETCH;
    m.item = -1;
    m.evals = 0;
    bool first = true;
    for (;;) {
        const float* eval_x = nullptr;
        float* eval_g = nullptr;
        // ---- warp-uniform control until the next evaluation is needed; the
        // states are tested in order of frequency (a line-search result after
        // nearly every evaluation, then the next BFGS iteration)
        while (eval_x == nullptr) {
            if (st == S_LS_DONE) {
                const float f1 = m.last_e;
                bool accept = (f1 - m.f0 < 0.0001f * m.alpha * m.pg);
                if (!accept) {
                    m.alpha *= 0.5f;
                    if (++m.trial < 10) {
                        conf_increment<kW>(c, c.s + m.bx_off, c.s + L.p, m.alpha, c.s + L.xnew);
                        eval_x = c.s + L.xnew;
                        eval_g = c.s + L.gnew;
                        continue;
                    }
                }
                // line search done (bfgs.h:120-141): y = g_new - g, x = x_new,
                // and the sums g.g, y.p (and y.y at the first iteration) in one
                // pass and one reduction (each the same per-lane terms and
                // shuffle tree as a separate dot product)
                const int n = 6 + c.T;
                float* g = c.s + L.g;
                float* gnew = c.s + L.gnew;
                float* y = c.s + L.y;
                float* H = c.s + L.h;
                float* p = c.s + L.p;
                float gg = 0.0f, yp = 0.0f, yy = 0.0f;
                for (int i = lane; i < n; i += kW) {
                    const float gi = g[i], yi = gnew[i] - gi;
                    y[i] = yi;
                    gg += gi * gi;
                    yp += yi * p[i];
                    yy += yi * yi;
                }
                m.f0 = f1;
                copyw<kW>(c, c.s + m.bx_off, c.s + L.xnew, 7 + c.T);
                if (m.iter == 0) lanes_sum3<kW>(gg, yp, yy);
                else lanes_sum2<kW>(gg, yp);
                if (!(sqrtf(gg) >= 1e-5f)) {
                    st = S_BFGS_END;
                    continue;
                }
                copyw<kW>(c, g, gnew, n);
                if (m.iter == 0 && fabsf(yy) > kEps) {
                    const float d = __fdividef(m.alpha * yp, yy);
                    for (int i = lane; i < n; i += kW) H[i * n + i] = d;
                    lanes_sync<kW>();
                }
                h_update<kW>(c, H, p, y, c.s + L.mhy, m.alpha, n, yp);
                ++m.iter;
                st = S_BFGS_ITER;
            } else if (st == S_BFGS_ITER) {
                if (m.iter >= m.steps_cap) {
                    st = S_BFGS_END;
                    continue;
                }
                const int n = 6 + c.T;
                float* p = c.s + L.p;
                m.pg = minus_hv_dot<kW>(c, c.s + L.h, c.s + L.g, p, c.s + L.g, n);
                m.alpha = 1.0f;
                m.trial = 0;
                conf_increment<kW>(c, c.s + m.bx_off, p, m.alpha, c.s + L.xnew);
                eval_x = c.s + L.xnew;
                eval_g = c.s + L.gnew;
                st = S_LS_DONE;
            } else if (st == S_FETCH) {
                int it;
                if constexpr (kStream) {  // (ligand, chain) of the next published item
                    int v[3] = {-1, 0, 0};
                    if (lane == 0) v[0] = stream_fetch(*SV, P.exhaustiveness, &v[1], &v[2]);
                    const int lig = __shfl_sync(lanes_mask<kW>(), v[0], 0, kW);
                    if (lig < 0) {
                        st = S_EXIT;
                        break;
                    }
                    m.item = __shfl_sync(lanes_mask<kW>(), v[1], 0, kW);
                    m.lig = lig;
                    m.chain = __shfl_sync(lanes_mask<kW>(), v[2], 0, kW);
                    first = false;
                    it = 0;
                } else if (!kSearch) {
                    it = first ? blockIdx.x * chains_in_block + slot_in_block : n_items;
                } else if (P.persistent) {
                    unsigned int v = 0;
                    if (lane == 0) v = atomicAdd(queue, 1u);
                    it = (int)__shfl_sync(lanes_mask<kW>(), v, 0, kW);
                } else {
                    it = first ? first_item + blockIdx.x * chains_in_block + slot_in_block : n_items + first_item;
                    if (it >= first_item + n_items) it = -1;
                    else it -= first_item;
                }
                first = false;
                if (!kStream && (it < 0 || it >= n_items)) {
                    st = S_EXIT;
                    break;
                }
                if (!kStream) m.item = it;
                if (kSearch) {
                    if (!kStream) {
                        const int gi = P.persistent ? it : it + first_item;
                        m.lig = order[gi / P.exhaustiveness];
                        m.chain = gi % P.exhaustiveness;
                    }
                    c = make_ctx<kW>(B, m.lig, sw, L);
                    rng.init(P.seed, (uint32_t)m.lig, (uint32_t)m.chain);
                    m.steps_cap = c.local_steps;
                    if (P.bfgs_cap > 0 && P.bfgs_cap < m.steps_cap) m.steps_cap = P.bfgs_cap;
                    float* tmp = c.s + L.tmp;
                    random_conf<kW>(c, rng, M, tmp);
                    copyw<kW>(c, c.s + L.best, tmp, 7 + c.T);
                    m.tmp_e = kMaxFl;
                    m.best_e = kMaxFl;
                    m.step = 0;
                    m.evals = 0;
                    // one evaluation of the start pose (result unused) leaves its
                    // coordinates for the first mutation's gyration radius
                    m.v = P.hunt_cap;
                    eval_x = tmp;
                    eval_g = c.s + L.gnew;
                    st = S_MC_STEP;
                } else {
                    m.lig = opt_lig[it];
                    c = make_ctx<kW>(B, m.lig, sw, L);
                    float* x = c.s + L.x;
                    for (int i = lane; i < 7 + c.T; i += kW) x[i] = poses[(size_t)it * pose_stride + i];
                    lanes_sync<kW>();
                    m.steps_cap = opt_steps > 0 ? opt_steps : c.local_steps;
                    m.mode = 2;
                    m.bx_off = L.x;
                    m.v = opt_v;
                    m.evals = 0;
                    st = S_BFGS_BEGIN;
                }
            } else if (st == S_MC_STEP) {
                if (m.step >= P.global_steps) {
                    st = S_DONE;
                    continue;
                }
                float* cand = c.s + L.cand;
                copyw<kW>(c, cand, c.s + L.tmp, 7 + c.T);
                mutate<kW>(c, L, rng, P.mutation_amplitude, cand);
                m.mode = 0;
                m.bx_off = L.cand;
                m.v = P.hunt_cap;
                st = S_BFGS_BEGIN;
            } else if (st == S_BFGS_BEGIN) {
                h_identity<kW>(c, c.s + L.h, 6 + c.T);
                eval_x = c.s + m.bx_off;
                eval_g = c.s + L.g;
                st = S_BFGS_INIT;
            } else if (st == S_BFGS_INIT) {
                m.f0 = m.last_e;
                m.f_orig = m.last_e;
                copyw<kW>(c, c.s + L.gorig, c.s + L.g, 6 + c.T);
                copyw<kW>(c, c.s + L.xorig, c.s + m.bx_off, 7 + c.T);
                m.iter = 0;
                st = S_BFGS_ITER;
            } else if (st == S_BFGS_END) {
                if (!(m.f0 <= m.f_orig)) {
                    m.f0 = m.f_orig;
                    copyw<kW>(c, c.s + m.bx_off, c.s + L.xorig, 7 + c.T);
                    copyw<kW>(c, c.s + L.g, c.s + L.gorig, 6 + c.T);
                }
                st = (m.mode == 0) ? S_AFTER_SEARCH : (m.mode == 1 ? S_AFTER_REFINE : S_DONE);
            } else if (st == S_AFTER_SEARCH) {
                const float cand_e = m.f0;
                int accept = 0;
                if (lane == 0) {
                    uint4 u = rng.next();
                    accept = (m.step == 0) || (cand_e < m.tmp_e) ||
                             (u01(u.x) < __expf(__fdividef(m.tmp_e - cand_e, P.temperature)));
                }
                accept = __shfl_sync(lanes_mask<kW>(), accept, 0, kW);
                if (accept) {
                    copyw<kW>(c, c.s + L.tmp, c.s + L.cand, 7 + c.T);
                    m.tmp_e = cand_e;
                    if (m.tmp_e < m.best_e) {
                        m.mode = 1;
                        m.bx_off = L.tmp;
                        m.v = P.authentic_v;
                        st = S_BFGS_BEGIN;
                        continue;
                    }
                }
                ++m.step;
                st = S_MC_STEP;
            } else if (st == S_AFTER_REFINE) {
                m.tmp_e = m.f0;
                if (m.tmp_e < m.best_e) {
                    copyw<kW>(c, c.s + L.best, c.s + L.tmp, 7 + c.T);
                    m.best_e = m.tmp_e;
                }
                ++m.step;
                st = S_MC_STEP;
            } else if (st == S_DONE) {
                if (kSearch) {
                    int slot = m.lig * P.exhaustiveness + m.chain;
                    unsigned sslot = 0;
                    if constexpr (kStream) {  // this slot's area of the result ring
                        sslot = (unsigned)m.item / ((unsigned)SV->slot_ligands * (unsigned)P.exhaustiveness);
                        const int local = m.lig - (int)sslot * SV->slot_ligands;
                        slot = ((int)(sslot % (unsigned)SV->ring) * SV->slot_ligands + local) * P.exhaustiveness +
                               m.chain;
                    }
                    const float* best = c.s + L.best;
                    for (int i = lane; i < 7 + c.T; i += kW) poses[(size_t)slot * pose_stride + i] = best[i];
                    // scoring-path energies of the best pose for the final rescoring
                    // (vina.h:241-300), so that post-processing needs no device work
                    float eg, ei;
                    eval_score<kAD4, kW>(c, L, M, Tb, best, P.authentic_v, eg, ei);
                    if (lane == 0) {
                        results[slot].e = m.best_e;
                        results[slot].evals = m.evals;
                        results[slot].ligand = m.lig;
                        results[slot].chain = m.chain;
                        results[slot].e_grid = eg;
                        results[slot].e_intra = ei;
                    }
                    if constexpr (kStream) {  // the slot's last chain tells the host
                        lanes_sync<kW>();
                        if (lane == 0) {
                            __threadfence();
                            if (atomicSub(SV->slot_left + sslot, 1u) == 1u) {
                                __threadfence_system();
                                *((volatile unsigned int*)(SV->done_host + sslot)) = 1u;
                            }
                        }
                    }
                } else {
                    const float* x = c.s + L.x;
                    for (int i = lane; i < 7 + c.T; i += kW) poses[(size_t)m.item * pose_stride + i] = x[i];
                    if (lane == 0) {
                        opt_e[m.item] = m.f0;
                        if (opt_evals) opt_evals[m.item] = m.evals;
                    }
                }
                lanes_sync<kW>();
                st = S_FETCH;
            } else {  // S_EXIT
                break;
            }
        }
        if (st == S_EXIT) return;
        // ---- the single evaluation site
        m.last_e = eval_deriv<false, kAD4, false, kW>(c, L, M, Tb, eval_x, eval_g, m.v, m.v);
        ++m.evals;
    }
}

// ---------------------------------------------------------------- kernels
// CTAs per SM the register budget is sized for: 7 x 128 threads leaves 72
// registers a thread (measured faster than 8 CTAs at 64 registers, which spill)
#ifndef UD_SEARCH_MIN_BLOCKS
#define UD_SEARCH_MIN_BLOCKS 7
#endif
// the AD4 instantiation (three maps per atom, three pair-table rows) keeps more
// values live: 6 CTAs, 80 registers a thread
#ifndef UD_SEARCH_MIN_BLOCKS_AD4
#define UD_SEARCH_MIN_BLOCKS_AD4 6
#endif
template <bool kAD4, int kW>
__global__ void __launch_bounds__(128, kAD4 ? UD_SEARCH_MIN_BLOCKS_AD4 : UD_SEARCH_MIN_BLOCKS) search_kernel(
    const __grid_constant__ Batch B, const __grid_constant__ Maps M, const __grid_constant__ Tables Tb,
    const __grid_constant__ SearchParams P, const __grid_constant__ Layout L, const int* order, int n_items,
    int first_item, unsigned int* queue, float* poses, int pose_stride, ChainResult* results) {
    extern __shared__ __align__(16) float smem[];
    float* sw = smem + (size_t)(threadIdx.x / kW) * L.total;
    run_machine<true, kAD4, kW>(B, M, Tb, P, L, sw, order, n_items, first_item, queue, poses, pose_stride, results,
                            nullptr, 0, 0.f, nullptr, nullptr);
}

// The persistent search of a streaming screen (StreamView): one warp per chain.
template <bool kAD4>
__global__ void __launch_bounds__(128, kAD4 ? UD_SEARCH_MIN_BLOCKS_AD4 : UD_SEARCH_MIN_BLOCKS) stream_kernel(
    const __grid_constant__ Batch B, const __grid_constant__ Maps M, const __grid_constant__ Tables Tb,
    const __grid_constant__ SearchParams P, const __grid_constant__ Layout L, const __grid_constant__ StreamView SV,
    float* poses, int pose_stride, ChainResult* results) {
    // The grid is one full wave (blocks per SM x SMs), so every SM starts
    // with its share of blocks; those on the SMs left to the per-slot
    // clustering and refinement kernels return at once.  (Fewer blocks would
    // not do: the block scheduler spreads them over all SMs, and the leftover
    // room on each may be too small for a post-processing CTA.)
    unsigned smid;
    asm("mov.u32 %0, %%smid;" : "=r"(smid));
    if (SV.reserve_every > 0 && smid % (unsigned)SV.reserve_every == 0) return;
    extern __shared__ __align__(16) float smem[];
    float* sw = smem + (size_t)(threadIdx.x / 32) * L.total;
    run_machine<true, kAD4, 32, true>(B, M, Tb, P, L, sw, nullptr, 0, 0, nullptr, poses, pose_stride, results,
                                      nullptr, 0, 0.f, nullptr, nullptr, &SV);
}

// Local optimisation from given poses (quasi_newton, quasi_newton.cpp:42-53):
// one warp per pose, BFGS at curl cap v; poses updated in place.
template <bool kAD4>
__global__ void __launch_bounds__(128) optimize_kernel(
    const __grid_constant__ Batch B, const __grid_constant__ Maps M, const __grid_constant__ Tables Tb,
    const __grid_constant__ SearchParams P, const __grid_constant__ Layout L, const int* pose_lig,
    float* poses, int pose_stride, int n_poses, int max_steps, float v, float* e_out, int* evals_out) {
    extern __shared__ __align__(16) float smem[];
    float* sw = smem + (size_t)(threadIdx.x >> 5) * L.total;
    run_machine<false, kAD4, 32>(B, M, Tb, P, L, sw, nullptr, n_poses, 0, nullptr, poses, pose_stride, nullptr,
                             pose_lig, max_steps, v, e_out, evals_out);
}

// Fixed poses: energy (search form, caps v_intra / v_inter) and gradient per pose.
template <bool kAD4>
__global__ void __launch_bounds__(128) score_kernel(
    const __grid_constant__ Batch B, const __grid_constant__ Maps M, const __grid_constant__ Tables Tb,
    const __grid_constant__ Layout L, const int* pose_lig, const float* poses, int pose_stride, int n_poses,
    float v_intra, float v_inter, float* e_out, float* g_out, int g_stride, float* score_out) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const int pose = blockIdx.x * (blockDim.x >> 5) + warp;
    if (pose >= n_poses) return;
    float* sw = smem + (size_t)warp * L.total;
    const Ctx c = make_ctx(B, pose_lig[pose], sw, L);
    float* x = sw + L.x;
    const int cs = 7 + c.T;
    for (int i = c.lane; i < cs; i += 32) x[i] = poses[(size_t)pose * pose_stride + i];
    __syncwarp();
    if (g_out) {
        float* g = sw + L.g;
        float e = eval_deriv<false, kAD4>(c, L, M, Tb, x, g, v_intra, v_inter);
        for (int i = c.lane; i < 6 + c.T; i += 32) g_out[(size_t)pose * g_stride + i] = g[i];
        if (c.lane == 0) e_out[pose] = e;
    }
    if (score_out) {
        float eg, ei;
        eval_score<kAD4>(c, L, M, Tb, x, v_inter, eg, ei);
        if (c.lane == 0) {
            score_out[2 * pose] = eg;
            score_out[2 * pose + 1] = ei;
        }
    }
}

// ---------------------------------------------------------------- receptor atoms
// Scoring against the receptor atoms instead of the maps, as the reference
// does after its search unless --no_refine (vina.h:232-300, vina.cpp:1168-1283).

// non_cache::within (non_cache.cpp:408-418): the heavy atoms of the last
// kinematics lie inside the box, with a margin of 1e-4.
__device__ __forceinline__ bool heavy_within(const Ctx& c, const Layout& L, const Receptor& R) {
    const float4* xyz = reinterpret_cast<const float4*>(c.s + L.coords);
    const float m = 1e-4f;
    bool ok = true;
    for (int a = c.lane; a < c.n_atoms; a += 32) {
        if (!((c.atom_packed(L, a) >> 16) & 1)) continue;
        const float4 x = xyz[a];
        if (x.x < R.begin[0] - m || x.x > R.end[0] + m || x.y < R.begin[1] - m || x.y > R.end[1] + m ||
            x.z < R.begin[2] - m || x.z > R.end[2] + m)
            ok = false;
    }
    return __all_sync(kFull, ok);
}

// Scoring-path energies: inter = non_cache::eval at slope 1e6 and cap v
// (non_cache.cpp:35-110), intra = model::evali at cap v.
__device__ __forceinline__ void eval_score_receptor(const Ctx& c, const Layout& L, const Receptor& R,
                                                    const Tables& Tb, const float* conf, float v, float& e_inter,
                                                    float& e_intra) {
    kinematics(c, L, conf);
    const float4* xyz = reinterpret_cast<const float4*>(c.s + L.coords);
    const BiasRec* bias;
    int n_bias;
    bias_of(R, c.lig, bias, n_bias);
    float ei = 0;
    for (int k = 0; k < c.n_grid; ++k) {
        const int a = c.grid_word(L, k) & 0xFF;
        const int t1 = ((c.atom_packed(L, a) >> 24) & 0xFF) - 1;
        float gx, gy, gz;
        ei += receptor_term<false>(R, Tb, t1, xyz[a], v, 1e6f, bias, n_bias, gx, gy, gz);
    }
    e_inter = ei;
    e_intra = intra_fast<false>(c, Tb, xyz, v);
}

// quasi_newton against the receptor atoms at out-of-box slope `slope`, curl
// caps v, from the conformation at L.x (updated in place): the iterations and
// line search of bfgs.h:63-146, as run_machine performs them.
__device__ float bfgs_receptor(const Ctx& c, const Layout& L, const Tables& Tb, const Receptor& R, int steps, float v,
                               float slope) {
    const Maps M{};
    const int n = 6 + c.T, cs = 7 + c.T;
    float* x = c.s + L.x;
    float* xnew = c.s + L.xnew;
    float* xorig = c.s + L.xorig;
    float* g = c.s + L.g;
    float* gnew = c.s + L.gnew;
    float* gorig = c.s + L.gorig;
    float* p = c.s + L.p;
    float* y = c.s + L.y;
    float* H = c.s + L.h;
    h_identity(c, H, n);
    float f0 = eval_deriv<false, false, true>(c, L, M, Tb, x, g, v, v, &R, slope);
    const float f_orig = f0;
    copyw(c, gorig, g, n);
    copyw(c, xorig, x, cs);
    for (int iter = 0; iter < steps; ++iter) {
        minus_hv(c, H, g, p, n);
        const float pg = dotw(c, p, g, n);
        float alpha = 1.0f, f1 = 0.0f;
        for (int trial = 0;;) {
            conf_increment(c, x, p, alpha, xnew);
            f1 = eval_deriv<false, false, true>(c, L, M, Tb, xnew, gnew, v, v, &R, slope);
            if (f1 - f0 < 0.0001f * alpha * pg) break;
            alpha *= 0.5f;
            if (++trial >= 10) break;
        }
        for (int i = c.lane; i < n; i += 32) y[i] = gnew[i] - g[i];
        __syncwarp();
        f0 = f1;
        copyw(c, x, xnew, cs);
        const float gg = dotw(c, g, g, n);
        if (!(sqrtf(gg) >= 1e-5f)) break;
        copyw(c, g, gnew, n);
        if (iter == 0) {
            const float yy = dotw(c, y, y, n);
            if (fabsf(yy) > kEps) {
                const float d = __fdividef(alpha * dotw(c, y, p, n), yy);
                for (int i = c.lane; i < n; i += 32) H[i * n + i] = d;
                __syncwarp();
            }
        }
        h_update(c, H, p, y, c.s + L.mhy, alpha, n, dotw(c, y, p, n));
    }
    if (!(f0 <= f_orig)) {
        f0 = f_orig;
        copyw(c, x, xorig, cs);
        copyw(c, g, gorig, n);
    }
    return f0;
}

// One warp per pose (pose_lig < 0: skipped); the modes of ReceptorMode.
// Refinement follows vina.h:251-272: up to refine_step rounds of quasi_newton
// (per-ligand (25 + atoms)/3 steps) at slopes 100, 1e4, 1e6, ..., stopping once
// the heavy atoms are inside the box.
template <int kMode>
__global__ void __launch_bounds__(128) receptor_kernel(
    const __grid_constant__ Batch B, const __grid_constant__ Tables Tb, const __grid_constant__ Receptor R,
    const __grid_constant__ Layout L, const int* pose_lig, float* poses, int pose_stride, int n_poses,
    int refine_step, float slope, float v, float* e_out, float* g_out, int g_stride, float4* out4) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const int pose = blockIdx.x * (blockDim.x >> 5) + warp;
    if (pose >= n_poses) return;
    const int lig = pose_lig[pose];
    if (lig < 0) return;
    float* sw = smem + (size_t)warp * L.total;
    const Ctx c = make_ctx(B, lig, sw, L);
    float* x = sw + L.x;
    const int cs = 7 + c.T;
    for (int i = c.lane; i < cs; i += 32) x[i] = poses[(size_t)pose * pose_stride + i];
    __syncwarp();
    if constexpr (kMode == kRecEnergyGrad) {
        const Maps M{};
        float* g = sw + L.g;
        const float e = eval_deriv<false, false, true>(c, L, M, Tb, x, g, v, v, &R, slope);
        for (int i = c.lane; i < 6 + c.T; i += 32) g_out[(size_t)pose * g_stride + i] = g[i];
        if (c.lane == 0) e_out[pose] = e;
    } else {
        float e_last = 0.0f;
        if constexpr (kMode == kRecRefine) {
            float sl = 100.0f;
            for (int r = 0; r < refine_step; ++r) {
                e_last = bfgs_receptor(c, L, Tb, R, c.local_steps, v, sl);
                kinematics(c, L, x);
                if (heavy_within(c, L, R)) break;
                sl *= 100.0f;
            }
            for (int i = c.lane; i < cs; i += 32) poses[(size_t)pose * pose_stride + i] = x[i];
        }
        float ei, ea;
        eval_score_receptor(c, L, R, Tb, x, v, ei, ea);
        const bool within = heavy_within(c, L, R);
        if (c.lane == 0) out4[pose] = make_float4(e_last, ei, ea, within ? 1.0f : 0.0f);
    }
}

// ---------------------------------------------------------------- bias wells on the maps
// cache::compute_bias (cache.cpp:789-957): at every map point, in list order,
// each well adds Vset exp(-d^2 / r^2) to the maps of the slots it reaches when
// that is below -0.01.  Probe points as the map build places them.
__global__ void __launch_bounds__(256) bias_maps_kernel(const BiasMapRec* __restrict__ bias, int n_bias, int nx, int ny,
                                                        int nz, int n_slots, float init0, float init1, float init2,
                                                        float finv0, float finv1, float finv2,
                                                        float* __restrict__ maps) {
    const size_t plane = (size_t)nx * ny * nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((size_t)nx * ny));
        const float px = __fadd_rn(init0, __fmul_rn(finv0, (float)x));
        const float py = __fadd_rn(init1, __fmul_rn(finv1, (float)y));
        const float pz = __fadd_rn(init2, __fmul_rn(finv2, (float)z));
        for (int k = 0; k < n_bias; ++k) {
            const BiasMapRec b = bias[k];
            const float dx = __fsub_rn(b.x, px), dy = __fsub_rn(b.y, py), dz = __fsub_rn(b.z, pz);
            const float rb2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
            const float dE = __fmul_rn(b.vset, expf(__fdiv_rn(__fdiv_rn(-rb2, b.r), b.r)));
            if (dE >= -0.01f) continue;
            for (int s = 0; s < n_slots; ++s) {
                const unsigned int word = s < 32 ? b.slots_lo : b.slots_hi;
                if ((word >> (s & 31)) & 1u) maps[(size_t)s * plane + i] = __fadd_rn(maps[(size_t)s * plane + i], dE);
            }
        }
    }
}

// ---------------------------------------------------------------- clustering
// Heavy-atom RMSD (rmsd_upper_bound, coords.cpp:28-35) between the current
// kinematics (or scratch slot `a`) and scratch slot `b`.
__device__ __forceinline__ float heavy_rmsd(const Ctx& c, const float4* xyz, const float* a, const float* b,
                                            int n_heavy) {
    float sum = 0;
    for (int i = c.lane; i < c.n_atoms; i += 32) {
        if (!((__ldg(&c.atoms()[i].packed) >> 16) & 1)) continue;
        float dx, dy, dz;
        if (a) {
            dx = a[3 * i] - b[3 * i]; dy = a[3 * i + 1] - b[3 * i + 1]; dz = a[3 * i + 2] - b[3 * i + 2];
        } else {
            const float4 p = xyz[i];
            dx = p.x - b[3 * i]; dy = p.y - b[3 * i + 1]; dz = p.z - b[3 * i + 2];
        }
        sum += dx * dx + dy * dy + dz * dz;
    }
    return sqrtf(warp_sum(sum) / (float)n_heavy);
}

// Stable insertion sort of slot ids by energy (lane 0).
__device__ __forceinline__ void sort_slots(int* ids, const float* e, int n) {
    if ((threadIdx.x & 31) == 0)
        for (int i = 1; i < n; ++i) {
            const int v = ids[i];
            int j = i - 1;
            while (j >= 0 && e[ids[j]] > e[v]) {
                ids[j + 1] = ids[j];
                --j;
            }
            ids[j + 1] = v;
        }
    __syncwarp();
}

// The modes of one ligand from its chains (warp per ligand): each chain's best
// pose goes through add_to_output_container (coords.cpp:44-68) in chain order
// with at most `cap` modes, then the modes through Vina::remove_redundant
// (vina.cpp:1465-1470).  The coordinates of the modes are kept in `scratch`.
__global__ void __launch_bounds__(128) cluster_kernel(
    const __grid_constant__ Batch B, const __grid_constant__ Layout L, const float* poses, int pose_stride,
    const ChainResult* results, int n_lig, int E, int cap, float min_rmsd, float* scratch, int max_atoms,
    int* n_modes, int* mode_chain, int* mode_lig, float* mode_pose) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const int lig = blockIdx.x * (blockDim.x >> 5) + warp;
    if (lig >= n_lig) return;
    const int cap4 = pad4(cap);
    float* sw = smem + (size_t)warp * (L.total + 4 * cap4);
    int* ord = reinterpret_cast<int*>(sw + L.total);
    float* ent_e = sw + L.total + cap4;
    int* ent_chain = reinterpret_cast<int*>(sw + L.total + 2 * cap4);
    int* keep = reinterpret_cast<int*>(sw + L.total + 3 * cap4);
    const Ctx c = make_ctx(B, lig, sw, L);
    const int n_heavy = __ldg(&B.ligs[lig].n_heavy);
    const float4* xyz = reinterpret_cast<const float4*>(c.s + L.coords);
    float* S = scratch + (size_t)lig * cap * 3 * max_atoms;
    const int cs = 7 + c.T;
    const float eps = 1.1920929e-7f;  // FLT_EPSILON
    int n = 0;
    for (int ch = 0; ch < E; ++ch) {
        const size_t item = (size_t)lig * E + ch;
        const float e = __ldg(&results[item].e);
        if (e < eps && e > -eps) continue;  // an energy of exactly 0 marks a failed chain
        float* x = c.s + L.x;
        for (int i = c.lane; i < cs; i += 32) x[i] = __ldg(poses + item * pose_stride + i);
        __syncwarp();
        kinematics(c, L, x);
        int best = n;
        float best_r = kMaxFl;
        for (int k = 0; k < n; ++k) {
            const float r = heavy_rmsd(c, xyz, nullptr, S + (size_t)ord[k] * 3 * max_atoms, n_heavy);
            if (k == 0 || r < best_r) {
                best = k;
                best_r = r;
            }
        }
        int slot = -1;
        if (best < n && best_r < min_rmsd) {
            if (e < ent_e[ord[best]]) slot = ord[best];
        } else if (n < cap) {
            slot = n;
            if (c.lane == 0) ord[n] = n;
            ++n;
        } else if (e < ent_e[ord[n - 1]]) {
            slot = ord[n - 1];
        }
        if (slot >= 0) {
            float* Sd = S + (size_t)slot * 3 * max_atoms;
            for (int a = c.lane; a < c.n_atoms; a += 32) {
                const float4 p = xyz[a];
                Sd[3 * a] = p.x; Sd[3 * a + 1] = p.y; Sd[3 * a + 2] = p.z;
            }
            if (c.lane == 0) {
                ent_e[slot] = e;
                ent_chain[slot] = ch;
            }
            __syncwarp();
            sort_slots(ord, ent_e, n);
        }
    }
    // remove_redundant: the modes in energy order into a fresh container
    int m = 0;
    for (int k = 0; k < n; ++k) {
        const int sl = ord[k];
        const float* Sa = S + (size_t)sl * 3 * max_atoms;
        int best = m;
        float best_r = kMaxFl;
        for (int j = 0; j < m; ++j) {
            const float r = heavy_rmsd(c, xyz, Sa, S + (size_t)keep[j] * 3 * max_atoms, n_heavy);
            if (j == 0 || r < best_r) {
                best = j;
                best_r = r;
            }
        }
        if (best < m && best_r < min_rmsd) {
            if (ent_e[sl] < ent_e[keep[best]] && c.lane == 0) keep[best] = sl;
        } else {
            if (c.lane == 0) keep[m] = sl;
            ++m;
        }
        __syncwarp();
        sort_slots(keep, ent_e, m);
    }
    if (c.lane == 0) n_modes[lig] = m;
    for (int k = 0; k < cap; ++k) {
        const size_t o = (size_t)lig * cap + k;
        const int ch = k < m ? ent_chain[keep[k]] : -1;
        if (c.lane == 0) {
            mode_chain[o] = ch;
            mode_lig[o] = k < m ? lig : -1;
        }
        if (k < m)
            for (int i = c.lane; i < cs; i += 32)
                mode_pose[o * pose_stride + i] = __ldg(poses + ((size_t)lig * E + ch) * pose_stride + i);
    }
}

// ---------------------------------------------------------------- adjoint
// Per-term data of the scoring function for weight gradients: the maps and the
// lerp rows of each unweighted term, laid out like the weighted ones.  Maps
// and tables are linear in the term weights, so a weighted map is the sum of
// the term maps times their weights.
constexpr int kMaxTerms = 6;
struct TermData {
    const float* maps;     // [term][slot][z][y][x]
    const float4* rows;    // [term][tp][bin] = (e, dor) of the bin and the next, as Tables::smooth4
    int n_terms;
    long long map_block;   // floats per term in `maps`
    long long row_block;   // float4 per term in `rows`
};

// Trilinear interpolation of one map at p, clamped to the box like grid_eval
// (grid.cpp:40-129) but without curl or out-of-box penalty; `cell` and `frac`
// cache the corner index and fractions for further maps of the same point.
__device__ __forceinline__ void grid_cell(const Maps& M, const float4 pos, int& cell, float* frac) {
    const int dims[3] = {M.nx, M.ny, M.nz};
    const float p[3] = {pos.x, pos.y, pos.z};
    int a[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float si = (p[i] - M.init[i]) * M.factor[i];
        if (si < 0) {
            a[i] = 0; si = 0;
        } else if (si >= M.dim_m1[i]) {
            a[i] = dims[i] - 2; si = 1;
        } else {
            a[i] = (int)si; si -= a[i];
        }
        frac[i] = si;
    }
    cell = a[0] + M.nx * (a[1] + M.ny * a[2]);
}

__device__ __forceinline__ float trilinear(const Maps& M, const float* g, int cell, const float* frac) {
    const int sy = M.nx, sz = M.nx * M.ny;
    const float x = frac[0], y = frac[1], z = frac[2];
    const float mx = 1 - x, my = 1 - y, mz = 1 - z;
    return __ldg(g + cell) * mx * my * mz + __ldg(g + cell + 1) * x * my * mz +
           __ldg(g + cell + sy) * mx * y * mz + __ldg(g + cell + 1 + sy) * x * y * mz +
           __ldg(g + cell + sz) * mx * my * z + __ldg(g + cell + 1 + sz) * x * my * z +
           __ldg(g + cell + sy + sz) * mx * y * z + __ldg(g + cell + 1 + sy + sz) * x * y * z;
}

// d curl(e) / d e for curl(e) = e v / (v + e) when e > 0 (curl.h:28-43)
__device__ __forceinline__ float curl_slope(float e, float v) {
    if (!(e > 0) || !(v < 0.1f * kMaxFl)) return 1.0f;
    const float t = (v < kEps) ? 0.0f : v / (v + e);
    return t * t;
}

// Fixed poses, differentiation form: energy (caps v_intra / v_inter), its
// gradient in the pose layout (d/dposition, d/dq, d/dtorsions; pair forces
// exact or as the reference's tables give them, see eval_deriv) and, when
// dw_out is set, its derivative with respect to each term weight.  The
// conformer is recomputed from the pose (forward kinematics) rather than
// stored.  The orientation gradient is 2 (0, tau) (x) q for the torque tau
// of a rotation applied on the left (quaternion_increment, quaternion.h), the
// gradient tangent to the unit sphere at a unit q.
template <bool kAD4>
__global__ void __launch_bounds__(128) adjoint_kernel(
    const __grid_constant__ Batch B, const __grid_constant__ Maps M, const __grid_constant__ Tables Tb,
    const __grid_constant__ Layout L, const __grid_constant__ TermData TD, int n_ligands, const int* pose_lig,
    const float* poses, int pose_stride, int n_poses, float v_intra, float v_inter, int exact, float* e_out,
    float* g_out, int g_stride, float* dw_out, int dw_stride) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const int pose = blockIdx.x * (blockDim.x >> 5) + warp;
    if (pose >= n_poses) return;
    const int lig = pose_lig[pose];
    const int lane = threadIdx.x & 31;
    if (lig < 0 || lig >= n_ligands) {  // refused pose: NaN outputs, no reads
        if (lane == 0) e_out[pose] = __int_as_float(0x7fc00000);
        return;
    }
    float* sw = smem + (size_t)warp * L.total;
    const Ctx c = make_ctx(B, lig, sw, L);
    float* x = sw + L.x;
    const int cs = 7 + c.T;
    for (int i = c.lane; i < cs; i += 32) x[i] = poses[(size_t)pose * pose_stride + i];
    __syncwarp();
    float* g = sw + L.g;
    const float e = exact ? eval_deriv<true, kAD4>(c, L, M, Tb, x, g, v_intra, v_inter)
                          : eval_deriv<false, kAD4>(c, L, M, Tb, x, g, v_intra, v_inter);
    if (c.lane == 0) e_out[pose] = e;
    if (g_out) {
        float* go = g_out + (size_t)pose * g_stride;
        if (c.lane == 0) {
            const float t0 = g[3], t1 = g[4], t2 = g[5];
            const float q0 = x[3], q1 = x[4], q2 = x[5], q3 = x[6];
            go[0] = g[0]; go[1] = g[1]; go[2] = g[2];
            go[3] = -2.0f * (t0 * q1 + t1 * q2 + t2 * q3);
            go[4] = 2.0f * (q0 * t0 + (t1 * q3 - t2 * q2));
            go[5] = 2.0f * (q0 * t1 + (t2 * q1 - t0 * q3));
            go[6] = 2.0f * (q0 * t2 + (t0 * q2 - t1 * q1));
        }
        for (int i = c.lane; i < c.T; i += 32) go[7 + i] = g[6 + i];
    }
    if (dw_out) {
        float acc[kMaxTerms];
#pragma unroll
        for (int t = 0; t < kMaxTerms; ++t) acc[t] = 0;
        const float4* xyz = reinterpret_cast<const float4*>(sw + L.coords);  // conformer of the evaluation above
        const size_t plane = (size_t)M.nx * M.ny * M.nz;
        for (int k = c.lane; k < c.n_grid; k += 32) {
            const uint32_t ga = c.grid_word(L, k);
            const int a = ga & 0xFF, slot = ga >> 8;
            int cell;
            float frac[3];
            grid_cell(M, xyz[a], cell, frac);
            const float w = curl_slope(trilinear(M, M.data + slot * plane, cell, frac), v_inter);
#pragma unroll
            for (int t = 0; t < kMaxTerms; ++t)
                if (t < TD.n_terms) acc[t] += w * trilinear(M, TD.maps + t * TD.map_block + slot * plane, cell, frac);
            if constexpr (kAD4) {
                const float q = __ldg(c.q() + a), aq = fabsf(q);
                const float we = q * curl_slope(trilinear(M, M.data + M.e_slot * plane, cell, frac), v_inter);
                const float wd = aq * curl_slope(trilinear(M, M.data + M.d_slot * plane, cell, frac), v_inter);
#pragma unroll
                for (int t = 0; t < kMaxTerms; ++t)
                    if (t < TD.n_terms) {
                        const float* tm = TD.maps + t * TD.map_block;
                        acc[t] += we * trilinear(M, tm + M.e_slot * plane, cell, frac) +
                                  wd * trilinear(M, tm + M.d_slot * plane, cell, frac);
                    }
            }
        }
        for (int k = c.lane; k < c.n_pairs; k += 32) {
            const uint32_t pr = __ldg(c.pairs() + k);
            if (pr == kPairPad) continue;
            const int a = pr & 0xFF, b = (pr >> 8) & 0xFF, tp = pr >> 16;
            const float4 pa = xyz[a], pb = xyz[b];
            const float rx = pb.x - pa.x, ry = pb.y - pa.y, rz = pb.z - pa.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            if (!(r2 < Tb.cutoff2)) continue;
            const float rf = Tb.factor * r2;
            const int i1 = (int)rf;
            const float rem = rf - i1;
            float4 row = __ldg(Tb.smooth4 + (size_t)tp * Tb.n_bins + i1);
            float2 cf = make_float2(0.f, 0.f);
            if constexpr (kAD4) {
                cf = __ldg(c.coef() + k);
                const float4 te = __ldg(Tb.smooth4 + (size_t)kAd4RowE * Tb.n_bins + i1);
                const float4 tg = __ldg(Tb.smooth4 + (size_t)kAd4RowG * Tb.n_bins + i1);
                row.x += cf.x * te.x + cf.y * tg.x;
                row.z += cf.x * te.z + cf.y * tg.z;
            }
            const float w = curl_slope(row.x + rem * (row.z - row.x), v_intra);
#pragma unroll
            for (int t = 0; t < kMaxTerms; ++t)
                if (t < TD.n_terms) {
                    const float4* tr = TD.rows + t * TD.row_block;
                    float4 rt = __ldg(tr + (size_t)tp * Tb.n_bins + i1);
                    if constexpr (kAD4) {
                        const float4 te = __ldg(tr + (size_t)kAd4RowE * Tb.n_bins + i1);
                        const float4 tg = __ldg(tr + (size_t)kAd4RowG * Tb.n_bins + i1);
                        rt.x += cf.x * te.x + cf.y * tg.x;
                        rt.z += cf.x * te.z + cf.y * tg.z;
                    }
                    acc[t] += w * (rt.x + rem * (rt.z - rt.x));
                }
        }
#pragma unroll
        for (int t = 0; t < kMaxTerms; ++t) acc[t] = warp_sum(acc[t]);
        if (c.lane == 0)
            for (int t = 0; t < TD.n_terms; ++t) dw_out[(size_t)pose * dw_stride + t] = acc[t];
    }
}

// Weighted sum of per-term blocks: out[i] = sum_t w[t] * in[t * block + i]
// (maps and tables from their unweighted terms, ud_maps_set_weights).
struct TermWeights {
    float w[kMaxTerms];
};
__global__ void combine_terms_kernel(const float4* __restrict__ in, long long block4, int n_terms,
                                     const __grid_constant__ TermWeights W, float4* __restrict__ out,
                                     long long n4) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4;
         i += (long long)gridDim.x * blockDim.x) {
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int t = 0; t < n_terms; ++t) {
            const float4 v = __ldg(in + t * block4 + i);
            const float wt = W.w[t];
            acc.x += wt * v.x; acc.y += wt * v.y; acc.z += wt * v.z; acc.w += wt * v.w;
        }
        out[i] = acc;
    }
}

// The x-pair copy of the maps: out[i] = (maps[i], maps[i + 1]) with x + 1
// clamped to the last point of the row (never read there: trilinear cells
// start at x <= nx - 2).
__global__ void map_xpairs_kernel(const float* __restrict__ maps, int nx, size_t n, float2* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % (size_t)nx);
        out[i] = make_float2(maps[i], maps[x + 1 < nx ? i + 1 : i]);
    }
}

// FP32 issue-rate probe: independent FMA chains, used to report the FP32
// roofline denominator measured on the running GPU.
__global__ void fp32_peak_kernel(float* out, int iters) {
    float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5,
          a6 = a0 + 6, a7 = a0 + 7;
    const float m = 0.9999999f, k = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fmaf(a0, m, k); a1 = fmaf(a1, m, k); a2 = fmaf(a2, m, k); a3 = fmaf(a3, m, k);
            a4 = fmaf(a4, m, k); a5 = fmaf(a5, m, k); a6 = fmaf(a6, m, k); a7 = fmaf(a7, m, k);
        }
    }
    float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 123.456f) out[0] = r;
}

// L2 read-bandwidth probe: every thread streams float4 words of an
// L2-resident buffer with L2-only loads (ld.global.cg: no L1 allocation, so
// each word is fetched from L2 every time), `reps` passes over the buffer,
// each pass starting at another offset so that no thread re-reads its own
// words back to back.  Used to report the L2 roofline denominator measured on
// the running GPU.
__global__ void __launch_bounds__(256) l2_read_kernel(const float4* __restrict__ buf, unsigned n4, int reps,
                                                      float* out) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const unsigned stride = gridDim.x * blockDim.x;
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    for (int r = 0; r < reps; ++r) {
        const unsigned shift = (unsigned)r * 7919u * 256u;
        for (unsigned i = t; i < n4; i += stride) {
            unsigned j = i + shift;
            j = j >= n4 ? j % n4 : j;
            const float4 v = __ldcg(buf + j);
            acc.x += v.x; acc.y += v.y; acc.z += v.z; acc.w += v.w;
        }
    }
    if (acc.x + acc.y + acc.z + acc.w == 123.456f) out[0] = acc.x;
}

// Grid maps.  Block = 8x4x4 grid points; receptor atoms within reach of the
// tile are compacted into shared memory in ascending index order so every
// point sums its contributions in the reference's order (cache.cpp:471-549,
// szv_grid.cpp:26-57); arithmetic uses explicit round-to-nearest intrinsics
// (no contraction) to reproduce the reference's FP32 sums.
constexpr int kMapTX = 8, kMapTY = 4, kMapTZ = 4;
constexpr int kMapThreads = kMapTX * kMapTY * kMapTZ;
constexpr int kMaxSlots = 36;
constexpr float kAd4ShortCut = 8.0f, kAd4LongCut = 20.48f, kAd4QsolvDev = 0.01097f;

// x^n by repeated multiplication from 1 (int_pow, int_pow.h)
__device__ __forceinline__ float ipow(float x, int n) {
    float p = 1.0f;
    for (int i = 0; i < n; ++i) p *= x;
    return p;
}

__global__ void __launch_bounds__(kMapThreads) maps_kernel(
    const float4* __restrict__ rec, int n_rec, const float* __restrict__ fastT, int n_bins,
    int n_slots_pad, int n_slots, float factor, float cutoff2, int nx, int ny, int nz,
    float init0, float init1, float init2, float finv0, float finv1, float finv2,
    float* __restrict__ out) {
    __shared__ float4 stage[kMapThreads];
    __shared__ int warp_cnt[kMapThreads / 32];
    const int tx = threadIdx.x % kMapTX, ty = (threadIdx.x / kMapTX) % kMapTY,
              tz = threadIdx.x / (kMapTX * kMapTY);
    const int gx0 = blockIdx.x * kMapTX, gy0 = blockIdx.y * kMapTY, gz0 = blockIdx.z * kMapTZ;
    const int x = gx0 + tx, y = gy0 + ty, z = gz0 + tz;
    // tile bounding box
    const float lo[3] = {init0 + finv0 * gx0, init1 + finv1 * gy0, init2 + finv2 * gz0};
    const float hi[3] = {init0 + finv0 * (gx0 + kMapTX - 1), init1 + finv1 * (gy0 + kMapTY - 1),
                         init2 + finv2 * (gz0 + kMapTZ - 1)};
    const float reach2 = cutoff2 * 1.0001f + 1e-3f;
    const float px = __fadd_rn(init0, __fmul_rn(finv0, (float)x));
    const float py = __fadd_rn(init1, __fmul_rn(finv1, (float)y));
    const float pz = __fadd_rn(init2, __fmul_rn(finv2, (float)z));
    float acc[kMaxSlots];
#pragma unroll
    for (int k = 0; k < kMaxSlots; ++k) acc[k] = 0.0f;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < n_rec; base += kMapThreads) {
        // order-preserving compaction of the next chunk of candidate atoms
        const int i = base + threadIdx.x;
        bool take = false;
        float4 a = make_float4(0, 0, 0, 0);
        if (i < n_rec) {
            a = rec[i];
            float d2 = 0;
            float cc[3] = {a.x, a.y, a.z};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float d = fmaxf(fmaxf(lo[k] - cc[k], cc[k] - hi[k]), 0.0f);
                d2 += d * d;
            }
            take = d2 <= reach2;
        }
        unsigned msk = __ballot_sync(kFull, take);
        if (lane == 0) warp_cnt[wid] = __popc(msk);
        __syncthreads();
        int off = 0, tot = 0;
        for (int w = 0; w < kMapThreads / 32; ++w) {
            if (w < wid) off += warp_cnt[w];
            tot += warp_cnt[w];
        }
        if (take) stage[off + __popc(msk & ((1u << lane) - 1))] = a;
        __syncthreads();
        if (x < nx && y < ny && z < nz) {
            for (int k = 0; k < tot; ++k) {
                float4 r = stage[k];
                float dx = __fsub_rn(r.x, px), dy = __fsub_rn(r.y, py), dz = __fsub_rn(r.z, pz);
                float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                if (r2 <= cutoff2) {
                    const int t1 = __float_as_int(r.w);
                    const int bin = (int)__fmul_rn(factor, r2);
                    const float4* row = reinterpret_cast<const float4*>(
                        fastT + ((size_t)t1 * n_bins + bin) * n_slots_pad);
#pragma unroll
                    for (int q = 0; q < kMaxSlots / 4; ++q) {
                        if (4 * q < n_slots) {
                            float4 v = __ldg(row + q);
                            acc[4 * q] = __fadd_rn(acc[4 * q], v.x);
                            acc[4 * q + 1] = __fadd_rn(acc[4 * q + 1], v.y);
                            acc[4 * q + 2] = __fadd_rn(acc[4 * q + 2], v.z);
                            acc[4 * q + 3] = __fadd_rn(acc[4 * q + 3], v.w);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    if (x < nx && y < ny && z < nz) {
        const size_t plane = (size_t)nx * ny * nz;
        const size_t idx = x + (size_t)nx * (y + (size_t)ny * z);
#pragma unroll
        for (int k = 0; k < kMaxSlots; ++k)
            if (k < n_slots) out[k * plane + idx] = acc[k];
    }
}

// ---------------------------------------------------------------- AD4 maps
// AutoDock 4.2 grid maps computed from the AD4 pair terms
// (potentials.h:346-486) at the exact probe-atom distances: one map per
// requested AD type (vdW + H-bond within 8 A, the charge-independent part of
// desolvation within 20.48 A), the electrostatic map per unit ligand charge
// and the desolvation map per unit |ligand charge| -- the three maps
// ad4cache::eval_deriv combines (ad4cache.cpp:227-269).  Receptor atoms of
// the tile are staged in shared memory; one thread per grid point.
__global__ void __launch_bounds__(kMapThreads) maps_ad4_kernel(
    const float4* __restrict__ rec, const int* __restrict__ rec_ad, int n_rec, const __grid_constant__ Ad4Params P,
    const __grid_constant__ Ad4MapSpec S, int nx, int ny, int nz, float init0, float init1, float init2,
    float finv0, float finv1, float finv2, float* __restrict__ out) {
    __shared__ float4 stage[kMapThreads];
    __shared__ int stage_ad[kMapThreads];
    __shared__ int warp_cnt[kMapThreads / 32];
    const int tx = threadIdx.x % kMapTX, ty = (threadIdx.x / kMapTX) % kMapTY,
              tz = threadIdx.x / (kMapTX * kMapTY);
    const int gx0 = blockIdx.x * kMapTX, gy0 = blockIdx.y * kMapTY, gz0 = blockIdx.z * kMapTZ;
    const int x = gx0 + tx, y = gy0 + ty, z = gz0 + tz;
    const float lo[3] = {init0 + finv0 * gx0, init1 + finv1 * gy0, init2 + finv2 * gz0};
    const float hi[3] = {init0 + finv0 * (gx0 + kMapTX - 1), init1 + finv1 * (gy0 + kMapTY - 1),
                         init2 + finv2 * (gz0 + kMapTZ - 1)};
    const float long2 = kAd4LongCut * kAd4LongCut, short2 = kAd4ShortCut * kAd4ShortCut;
    const float reach2 = long2 * 1.0001f + 1e-3f;
    const float px = init0 + finv0 * (float)x, py = init1 + finv1 * (float)y, pz = init2 + finv2 * (float)z;
    float vh[kMaxSlots];
#pragma unroll
    for (int k = 0; k < kMaxSlots; ++k) vh[k] = 0.0f;
    float sum_vg = 0.0f, sum_sg = 0.0f, sum_qe = 0.0f;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < n_rec; base += kMapThreads) {
        const int i = base + threadIdx.x;
        bool take = false;
        float4 a = make_float4(0, 0, 0, 0);
        int aad = 0;
        if (i < n_rec) {
            a = rec[i];
            aad = rec_ad[i];
            float d2 = 0;
            const float cc[3] = {a.x, a.y, a.z};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float d = fmaxf(fmaxf(lo[k] - cc[k], cc[k] - hi[k]), 0.0f);
                d2 += d * d;
            }
            take = d2 <= reach2;
        }
        const unsigned msk = __ballot_sync(kFull, take);
        if (lane == 0) warp_cnt[wid] = __popc(msk);
        __syncthreads();
        int off = 0, tot = 0;
        for (int w = 0; w < kMapThreads / 32; ++w) {
            if (w < wid) off += warp_cnt[w];
            tot += warp_cnt[w];
        }
        if (take) {
            const int at = off + __popc(msk & ((1u << lane) - 1));
            stage[at] = a;
            stage_ad[at] = aad;
        }
        __syncthreads();
        if (x < nx && y < ny && z < nz) {
            for (int k = 0; k < tot; ++k) {
                const float4 r = stage[k];
                const float dx = r.x - px, dy = r.y - py, dz = r.z - pz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (!(r2 < long2)) continue;
                const float d = sqrtf(r2);
                const int ra = stage_ad[k];
                const float q = r.w;
                // desolvation distance factor and electrostatics (cutoff 20.48 A)
                const float xg = d / 3.6f;
                const float g = expf(-0.5f * (xg * xg));
                sum_vg += P.volume[ra] * g;
                sum_sg += (P.solvation[ra] + kAd4QsolvDev * fabsf(q)) * g;
                const float B = 78.4f + 8.5525f;
                const float diel = -8.5525f + B / (1.0f + 7.7839f * expf(-B * 0.003627f * d));
                const float einv = d < kEps ? 100.0f / diel : fminf(100.0f, 1.0f / (d * diel));
                sum_qe += q * 332.0f * einv;
                if (!(r2 < short2)) continue;
#pragma unroll
                for (int s = 0; s < kMaxSlots; ++s) {
                    if (s >= S.n_slots) break;
                    const int t = S.slot_ad[s];
                    const float hbd = P.hb_depth[t] * P.hb_depth[ra];
                    float rij, c_a, c_b;
                    int pa, pb;
                    if (hbd < 0) {  // H-bond 12-10
                        rij = P.hb_radius[t] + P.hb_radius[ra];
                        const float r10 = ipow(rij, 10);
                        c_a = ipow(rij, 12) * -hbd * 10.0f / 2.0f;
                        c_b = r10 * -hbd * 12.0f / 2.0f;
                        pa = 12;
                        pb = 10;
                    } else {  // vdW 12-6
                        rij = P.radius[t] + P.radius[ra];
                        const float depth = sqrtf(P.depth[t] * P.depth[ra]);
                        c_a = ipow(rij, 12) * depth;
                        c_b = ipow(rij, 6) * depth * 2.0f;
                        pa = 12;
                        pb = 6;
                    }
                    float rs = d;  // smoothing 0.5
                    if (rs > rij + 0.25f) rs -= 0.25f;
                    else if (rs < rij - 0.25f) rs += 0.25f;
                    else rs = rij;
                    const float ra_ = ipow(rs, pa), rb_ = ipow(rs, pb);
                    const float w = hbd < 0 ? S.w_hb : S.w_vdw;
                    const float e = (ra_ > kEps && rb_ > kEps) ? fminf(100000.0f, c_a / ra_ - c_b / rb_) : 100000.0f;
                    vh[s] += w * e;
                }
            }
        }
        __syncthreads();
    }
    if (x < nx && y < ny && z < nz) {
        const size_t plane = (size_t)nx * ny * nz;
        const size_t idx = x + (size_t)nx * (y + (size_t)ny * z);
#pragma unroll
        for (int s = 0; s < kMaxSlots; ++s)
            if (s < S.n_slots) {
                const int t = S.slot_ad[s];
                out[s * plane + idx] = vh[s] + S.w_dsolv * (P.solvation[t] * sum_vg + P.volume[t] * sum_sg);
            }
        out[S.n_slots * plane + idx] = S.w_elec * sum_qe;
        out[(S.n_slots + 1) * plane + idx] = S.w_dsolv * kAd4QsolvDev * sum_vg;
    }
}

}  // namespace dev

// ---------------------------------------------------------------- host side
// Launch helpers called from the C-ABI layer (ud_capi.cpp), declared in
// ud_engine.h with the device views they take.

static dev::Maps to_maps(const DeviceMapsView& m) {
    dev::Maps M;
    M.data = m.data;
    M.xp = m.xpairs;
    M.nx = m.desc.dims[0];
    M.ny = m.desc.dims[1];
    M.nz = m.desc.dims[2];
    for (int i = 0; i < 3; ++i) {
        M.init[i] = m.desc.init[i];
        M.factor[i] = m.desc.factor[i];
        M.factor_inv[i] = m.desc.factor_inv[i];
        M.dim_m1[i] = m.desc.dim_m1[i];
        M.corner2[i] = m.desc.corner2[i];
    }
    M.slope = m.desc.slope;
    M.e_slot = m.desc.e_slot;
    M.d_slot = m.desc.d_slot;
    return M;
}

static dev::Tables to_tables(const DeviceTablesView& t) {
    dev::Tables T;
    T.smooth4 = reinterpret_cast<const float4*>(t.smooth);
    T.fast = t.fast;
    T.n_bins = t.n_bins;
    T.factor = t.factor;
    T.cutoff2 = t.cutoff2;
    return T;
}

static dev::Batch to_batch(const DeviceBatchView& b) {
    dev::Batch B;
    B.ligs = b.ligs;
    B.atoms = b.atoms;
    B.nodes = b.nodes;
    B.pairs = b.pairs;
    B.grid_list = b.grid_list;
    B.charges = b.charges;
    B.pair_coef = reinterpret_cast<const float2*>(b.pair_coef);
    return B;
}

static dev::Receptor to_receptor(const DeviceReceptorView& r) {
    dev::Receptor R;
    R.atoms = reinterpret_cast<const float4*>(r.atoms);
    R.start = r.start;
    for (int i = 0; i < 3; ++i) {
        R.n[i] = r.n[i];
        R.begin[i] = r.begin[i];
        R.end[i] = r.end[i];
    }
    R.inv_cell = r.inv_cell;
    R.bias = r.bias;
    R.n_bias = r.n_bias;
    R.lig_bias = r.lig_bias;
    R.lig_bias_span = r.lig_bias_span;
    return R;
}

int engine_chain_smem_bytes(int max_atoms, int max_torsions) {
    return dev::make_layout(max_atoms, max_torsions).total * (int)sizeof(float);
}

cudaError_t launch_maps(const float* rec_xyzt, int n_rec, const float* fastT, int n_bins,
                        int n_slots, int n_slots_pad, float factor, float cutoff2,
                        const MapsDesc& d, float* out, cudaStream_t stream) {
    dim3 block(dev::kMapThreads);
    dim3 grid((d.dims[0] + dev::kMapTX - 1) / dev::kMapTX, (d.dims[1] + dev::kMapTY - 1) / dev::kMapTY,
              (d.dims[2] + dev::kMapTZ - 1) / dev::kMapTZ);
    dev::maps_kernel<<<grid, block, 0, stream>>>(
        reinterpret_cast<const float4*>(rec_xyzt), n_rec, fastT, n_bins, n_slots_pad, n_slots, factor,
        cutoff2, d.dims[0], d.dims[1], d.dims[2], d.init[0], d.init[1], d.init[2], d.factor_inv[0],
        d.factor_inv[1], d.factor_inv[2], out);
    return cudaGetLastError();
}

cudaError_t launch_maps_ad4(const float* rec_xyzq, const int* rec_ad, int n_rec, const Ad4Params& params,
                            const Ad4MapSpec& spec, const MapsDesc& d, float* out, cudaStream_t stream) {
    if (spec.n_slots < 0 || spec.n_slots > dev::kMaxSlots) return cudaErrorInvalidValue;
    dim3 block(dev::kMapThreads);
    dim3 grid((d.dims[0] + dev::kMapTX - 1) / dev::kMapTX, (d.dims[1] + dev::kMapTY - 1) / dev::kMapTY,
              (d.dims[2] + dev::kMapTZ - 1) / dev::kMapTZ);
    dev::maps_ad4_kernel<<<grid, block, 0, stream>>>(reinterpret_cast<const float4*>(rec_xyzq), rec_ad, n_rec, params,
                                                     spec, d.dims[0], d.dims[1], d.dims[2], d.init[0], d.init[1],
                                                     d.init[2], d.factor_inv[0], d.factor_inv[1], d.factor_inv[2], out);
    return cudaGetLastError();
}

cudaError_t launch_map_xpairs(const float* maps, const MapsDesc& d, float2* out, cudaStream_t stream) {
    const size_t n = (size_t)d.dims[0] * d.dims[1] * d.dims[2] * (size_t)d.n_maps;
    if (n == 0) return cudaSuccess;
    int dev_id = 0, n_sm = 148;
    cudaGetDevice(&dev_id);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev_id);
    const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)n_sm * 8);
    dev::map_xpairs_kernel<<<blocks, 256, 0, stream>>>(maps, d.dims[0], n, out);
    return cudaGetLastError();
}

// Dynamic shared memory allowed for kernel `fn` on the current device, raised
// to `smem` when below it and never lowered: a kernel launch captured in a graph earlier may need
// more than the launch at hand (another batch's layout), and the attribute is
// a per-kernel limit that later launches of the graph are checked against.
static cudaError_t smem_attr(const void* fn, size_t smem) {
    static std::mutex mu;
    static std::unordered_map<uint64_t, size_t> allowed;  // (kernel, device) -> bytes
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = allowed[(uint64_t)(uintptr_t)fn * 64u + (uint64_t)dev];
    if (smem <= cur) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) cur = smem;
    return e;
}

cudaError_t launch_score(const DeviceBatchView& b, const DeviceMapsView& m,
                         const DeviceTablesView& t, const int* pose_lig, const float* poses,
                         int pose_stride, int n_poses, float v_intra, float v_inter, float* e_out,
                         float* g_out, int g_stride, float* score_out, cudaStream_t stream) {
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    const int warps = 4;
    size_t smem = (size_t)warps * L.total * sizeof(float);
    const auto kern = m.desc.ad4 ? dev::score_kernel<true> : dev::score_kernel<false>;
    cudaError_t e = smem_attr((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((n_poses + warps - 1) / warps);
    kern<<<grid, warps * 32, smem, stream>>>(to_batch(b), to_maps(m), to_tables(t), L,
                                                          pose_lig, poses, pose_stride, n_poses,
                                                          v_intra, v_inter, e_out, g_out, g_stride,
                                                          score_out);
    return cudaGetLastError();
}

cudaError_t launch_adjoint(const DeviceBatchView& b, const DeviceMapsView& m, const DeviceTablesView& t,
                           const DeviceTermsView& terms, int n_ligands, const int* pose_lig, const float* poses,
                           int pose_stride, int n_poses, float v_intra, float v_inter, int exact, float* e_out,
                           float* g_out, int g_stride, float* dw_out, int dw_stride, cudaStream_t stream) {
    if (terms.n_terms > dev::kMaxTerms) return cudaErrorInvalidValue;
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    const int warps = 4;
    size_t smem = (size_t)warps * L.total * sizeof(float);
    const auto kern = m.desc.ad4 ? dev::adjoint_kernel<true> : dev::adjoint_kernel<false>;
    cudaError_t e = smem_attr((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    dev::TermData TD;
    TD.maps = terms.maps;
    TD.rows = reinterpret_cast<const float4*>(terms.rows);
    TD.n_terms = terms.n_terms;
    TD.map_block = terms.map_block;
    TD.row_block = terms.row_block;
    dim3 grid((n_poses + warps - 1) / warps);
    kern<<<grid, warps * 32, smem, stream>>>(to_batch(b), to_maps(m), to_tables(t), L, TD,
                                                            n_ligands, pose_lig, poses, pose_stride, n_poses,
                                                            v_intra, v_inter, exact, e_out, g_out, g_stride, dw_out,
                                                            dw_stride);
    return cudaGetLastError();
}

cudaError_t launch_combine_terms(const float* in, long long block, int n_terms, const float* w, float* out,
                                 cudaStream_t stream) {
    if (n_terms < 1 || n_terms > dev::kMaxTerms || (block & 3) != 0) return cudaErrorInvalidValue;
    if ((reinterpret_cast<uintptr_t>(in) & 15) != 0 || (reinterpret_cast<uintptr_t>(out) & 15) != 0)
        return cudaErrorMisalignedAddress;
    dev::TermWeights W{};
    for (int t = 0; t < n_terms; ++t) W.w[t] = w[t];
    const long long n4 = block / 4;
    int dev_id = 0, n_sm = 148;
    cudaGetDevice(&dev_id);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev_id);
    const long long want = (n4 + 255) / 256;
    const int blocks = (int)std::max<long long>(1, std::min<long long>(want, (long long)n_sm * 8));
    dev::combine_terms_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<const float4*>(in), n4, n_terms, W,
                                                         reinterpret_cast<float4*>(out), n4);
    return cudaGetLastError();
}

// The search kernel instantiation for the scoring function and the lanes a
// chain runs on (a warp, or half a warp).
using SearchKernel = void (*)(const dev::Batch, const dev::Maps, const dev::Tables, const SearchParams,
                              const dev::Layout, const int*, int, int, unsigned int*, float*, int, ChainResult*);
static SearchKernel search_kernel_for(bool ad4, int lanes) {
    if (lanes == 16) return ad4 ? dev::search_kernel<true, 16> : dev::search_kernel<false, 16>;
    return ad4 ? dev::search_kernel<true, 32> : dev::search_kernel<false, 32>;
}

cudaError_t launch_search(const DeviceBatchView& b, const DeviceMapsView& m,
                          const DeviceTablesView& t, const SearchParams& P, const int* order,
                          int n_items, int first_item, unsigned int* queue, float* poses,
                          int pose_stride, ChainResult* results, int grid_blocks,
                          cudaStream_t stream) {
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    if (P.chains_per_block < 1 || P.chains_per_block > 4 || (P.lanes_per_chain != 32 && P.lanes_per_chain != 16))
        return cudaErrorInvalidValue;
    const int warps = P.chains_per_block;                        // warps per CTA
    const int chains = warps * (32 / P.lanes_per_chain);         // chains per CTA
    size_t smem = (size_t)chains * L.total * sizeof(float);
    const auto kern = search_kernel_for(m.desc.ad4 != 0, P.lanes_per_chain);
    cudaError_t e = smem_attr((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    dim3 grid;
    if (P.persistent) grid = dim3(grid_blocks);
    else grid = dim3((n_items + chains - 1) / chains);
    kern<<<grid, warps * 32, smem, stream>>>(to_batch(b), to_maps(m), to_tables(t), P, L,
                                                           order, n_items, first_item, queue, poses,
                                                           pose_stride, results);
    return cudaGetLastError();
}

cudaError_t launch_search_stream(const DeviceBatchView& b, const DeviceMapsView& m, const DeviceTablesView& t,
                                 const SearchParams& P, const StreamView& sv, float* poses, int pose_stride,
                                 ChainResult* results, int blocks, cudaStream_t stream) {
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    if (P.chains_per_block < 1 || P.chains_per_block > 4 || blocks < 1) return cudaErrorInvalidValue;
    const int warps = P.chains_per_block;
    size_t smem = (size_t)warps * L.total * sizeof(float);
    const auto kern = b.ad4 ? dev::stream_kernel<true> : dev::stream_kernel<false>;
    cudaError_t e = smem_attr((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    kern<<<blocks, warps * 32, smem, stream>>>(to_batch(b), to_maps(m), to_tables(t), P, L, sv, poses, pose_stride,
                                               results);
    return cudaGetLastError();
}

// CTAs of the streaming kernel resident per SM at this layout and CTA size.
int stream_blocks_per_sm(const DeviceBatchView& b, int warps) {
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    size_t smem = (size_t)warps * L.total * sizeof(float);
    const auto kern = b.ad4 ? dev::stream_kernel<true> : dev::stream_kernel<false>;
    int nb = 0;
    if (smem_attr((const void*)kern, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, warps * 32, smem) != cudaSuccess) {
        cudaGetLastError();  // a CTA this size does not fit: no error left behind for the next launch
        return 0;
    }
    return nb;
}

cudaError_t launch_optimize(const DeviceBatchView& b, const DeviceMapsView& m,
                            const DeviceTablesView& t, const int* pose_lig, float* poses,
                            int pose_stride, int n_poses, int max_steps, float v, float* e_out,
                            int* evals_out, cudaStream_t stream) {
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    const int warps = 4;
    size_t smem = (size_t)warps * L.total * sizeof(float);
    const auto kern = m.desc.ad4 ? dev::optimize_kernel<true> : dev::optimize_kernel<false>;
    cudaError_t e = smem_attr((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    SearchParams P{};
    dim3 grid((n_poses + warps - 1) / warps);
    kern<<<grid, warps * 32, smem, stream>>>(to_batch(b), to_maps(m), to_tables(t), P, L,
                                                             pose_lig, poses, pose_stride, n_poses,
                                                             max_steps, v, e_out, evals_out);
    return cudaGetLastError();
}

cudaError_t launch_bias_maps(const BiasMapRec* bias, int n_bias, const MapsDesc& d, float* maps,
                             cudaStream_t stream) {
    if (n_bias <= 0) return cudaSuccess;
    const size_t plane = (size_t)d.dims[0] * d.dims[1] * d.dims[2];
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((plane + threads - 1) / threads, 148 * 16);
    dev::bias_maps_kernel<<<blocks, threads, 0, stream>>>(bias, n_bias, d.dims[0], d.dims[1], d.dims[2], d.n_maps,
                                                          d.init[0], d.init[1], d.init[2], d.factor_inv[0],
                                                          d.factor_inv[1], d.factor_inv[2], maps);
    return cudaGetLastError();
}

cudaError_t launch_cluster(const DeviceBatchView& b, const float* poses, int pose_stride, const ChainResult* results,
                           int n_ligands, int exhaustiveness, int cap, float min_rmsd, float* scratch, int* n_modes,
                           int* mode_chain, int* mode_lig, float* mode_pose, cudaStream_t stream) {
    if (n_ligands <= 0) return cudaSuccess;
    if (cap < 1) return cudaErrorInvalidValue;
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    const int warps = 4;
    size_t smem = (size_t)warps * (L.total + 4 * dev::pad4(cap)) * sizeof(float);
    cudaError_t e = smem_attr((const void*)dev::cluster_kernel, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((n_ligands + warps - 1) / warps);
    dev::cluster_kernel<<<grid, warps * 32, smem, stream>>>(to_batch(b), L, poses, pose_stride, results, n_ligands,
                                                            exhaustiveness, cap, min_rmsd, scratch, b.max_atoms,
                                                            n_modes, mode_chain, mode_lig, mode_pose);
    return cudaGetLastError();
}

cudaError_t prepare_stream_post(const DeviceBatchView& b, int cap, bool refine) {
    const dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    const int warps = 4;
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, (const void*)dev::cluster_kernel);
    if (e == cudaSuccess)
        e = smem_attr((const void*)dev::cluster_kernel, (size_t)warps * (L.total + 4 * dev::pad4(cap)) * sizeof(float));
    if (e != cudaSuccess || !refine) return e;
    const void* fn = (const void*)dev::receptor_kernel<kRecRefine>;
    e = cudaFuncGetAttributes(&fa, fn);
    if (e == cudaSuccess) e = smem_attr(fn, (size_t)warps * L.total * sizeof(float));
    return e;
}
cudaError_t launch_receptor(int mode, const DeviceBatchView& b, const DeviceTablesView& t,
                            const DeviceReceptorView& r, const int* pose_lig, float* poses, int pose_stride,
                            int n_poses, int refine_step, float slope, float v, float* e_out, float* g_out,
                            int g_stride, float* out4, cudaStream_t stream) {
    if (n_poses <= 0) return cudaSuccess;
    if (b.ad4) return cudaErrorInvalidValue;  // receptor-atom scoring is for Vina / Vinardo maps
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    const int warps = 4;
    size_t smem = (size_t)warps * L.total * sizeof(float);
    const void* fn = mode == kRecEnergyGrad ? (const void*)dev::receptor_kernel<kRecEnergyGrad>
                     : mode == kRecRefine   ? (const void*)dev::receptor_kernel<kRecRefine>
                                            : (const void*)dev::receptor_kernel<kRecScore>;
    cudaError_t e = smem_attr(fn, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((n_poses + warps - 1) / warps);
    const dev::Batch B = to_batch(b);
    const dev::Tables T = to_tables(t);
    const dev::Receptor R = to_receptor(r);
    float4* o4 = reinterpret_cast<float4*>(out4);
    if (mode == kRecEnergyGrad)
        dev::receptor_kernel<kRecEnergyGrad><<<grid, warps * 32, smem, stream>>>(
            B, T, R, L, pose_lig, poses, pose_stride, n_poses, refine_step, slope, v, e_out, g_out, g_stride, o4);
    else if (mode == kRecRefine)
        dev::receptor_kernel<kRecRefine><<<grid, warps * 32, smem, stream>>>(
            B, T, R, L, pose_lig, poses, pose_stride, n_poses, refine_step, slope, v, e_out, g_out, g_stride, o4);
    else
        dev::receptor_kernel<kRecScore><<<grid, warps * 32, smem, stream>>>(
            B, T, R, L, pose_lig, poses, pose_stride, n_poses, refine_step, slope, v, e_out, g_out, g_stride, o4);
    return cudaGetLastError();
}

// Measured FP32 FMA throughput (TFLOP/s) of the current device.
float measure_fp32_peak_tflops() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float* out = nullptr;
    if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) return 0;
    const int blocks = sms * 8, threads = 256, iters = 4096;
    dev::fp32_peak_kernel<<<blocks, threads>>>(out, 16);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 0;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(a);
        dev::fp32_peak_kernel<<<blocks, threads>>>(out, iters);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        best = std::max(best, (float)(flops / (ms * 1e-3) / 1e12));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    return best;
}

// Measured L2 read bandwidth (GB/s) of the current device: a 32 MB buffer
// (a quarter of the 126 MB L2) written once, then read 64 times over per
// launch by 8 CTAs of 256 threads per SM; best of 5 launches timed with CUDA
// events.
float measure_l2_read_gbs() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t bytes = 32u << 20;
    const unsigned n4 = (unsigned)(bytes / sizeof(float4));
    float4* buf = nullptr;
    float* out = nullptr;
    if (cudaMalloc(&buf, bytes) != cudaSuccess) return 0;
    if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) {
        cudaFree(buf);
        return 0;
    }
    cudaMemset(buf, 0, bytes);
    const int blocks = sms * 8, threads = 256, reps = 64;
    dev::l2_read_kernel<<<blocks, threads>>>(buf, n4, 2, out);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(a);
        dev::l2_read_kernel<<<blocks, threads>>>(buf, n4, reps, out);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms > 0) best = std::max(best, (float)((double)bytes * reps / (ms * 1e-3) / 1e9));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const bool ok = cudaGetLastError() == cudaSuccess;
    cudaFree(out);
    cudaFree(buf);
    return ok ? best : 0.0f;
}

int search_blocks_per_sm(const DeviceBatchView& b, int warps, int lanes_per_chain) {
    dev::Layout L = dev::make_layout(b.max_atoms, b.max_torsions);
    const int lanes = lanes_per_chain == 16 ? 16 : 32;
    size_t smem = (size_t)warps * (32 / lanes) * L.total * sizeof(float);
    const auto kern = search_kernel_for(b.ad4 != 0, lanes);
    int nb = 0;
    if (smem_attr((const void*)kern, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, warps * 32, smem) != cudaSuccess) {
        cudaGetLastError();  // a CTA this size does not fit: no error left behind for the next launch
        return 0;
    }
    return nb;
}

// ---------------------------------------------------------------- allocation-free search
// Scratch of the persistent search for callers that cannot allocate device
// memory when they search: a file-scope device array that every GPU loading
// the library holds until the process exits.  Layout: the work-queue counter
// (256 bytes), then one ChainResult per chain (kNoAllocMaxChains).  Every
// call shares it: the counter is cleared on each call, and calls that overlap
// on the GPU race on it.
constexpr size_t kNoAllocResultsOff = 256;
constexpr size_t kNoAllocBytes = kNoAllocResultsOff + (size_t)kNoAllocMaxChains * sizeof(ChainResult);
// the size the header and the design notes state (3,145,984 bytes, about 3.1 MB)
static_assert(kNoAllocBytes == 3145984, "documented scratch size");
static __device__ __align__(256) unsigned char g_search_scratch[kNoAllocBytes];

namespace dev {
__global__ void chain_results_out(const ChainResult* r, int n, float* e, int* evals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (e) e[i] = r[i].e;
    if (evals) evals[i] = r[i].evals;
}
}  // namespace dev

// Device address of g_search_scratch on the current device, looked up once per
// device (host code only holds a stand-in for the array, not its address).
// Threads racing on a device's first lookup store the same address.
static cudaError_t noalloc_scratch(unsigned char** out) {
    constexpr int kMaxDevices = 64;
    static std::atomic<unsigned char*> addr[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    unsigned char* p = addr[dev].load(std::memory_order_acquire);
    if (!p) {
        void* q = nullptr;
        e = cudaGetSymbolAddress(&q, g_search_scratch);
        if (e != cudaSuccess) return e;
        p = static_cast<unsigned char*>(q);
        addr[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return cudaSuccess;
}

cudaError_t launch_search_noalloc(const DeviceBatchView& b, const DeviceMapsView& m,
                                  const DeviceTablesView& t, const SearchParams& P,
                                  const int* d_order, int n_ligands, int grid_blocks, float* poses,
                                  int pose_stride, float* e_out, int* evals_out, cudaStream_t stream) {
    if ((long long)n_ligands * P.exhaustiveness > kNoAllocMaxChains) return cudaErrorInvalidValue;
    unsigned char* base = nullptr;
    cudaError_t e = noalloc_scratch(&base);
    if (e != cudaSuccess) return e;
    unsigned int* queue = reinterpret_cast<unsigned int*>(base);
    ChainResult* results = reinterpret_cast<ChainResult*>(base + kNoAllocResultsOff);
    const int n_items = n_ligands * P.exhaustiveness;
    e = cudaMemsetAsync(queue, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    SearchParams sp = P;
    sp.persistent = 1;
    e = launch_search(b, m, t, sp, d_order, n_items, 0, queue, poses, pose_stride, results, grid_blocks, stream);
    if (e != cudaSuccess) return e;
    dev::chain_results_out<<<(n_items + 255) / 256, 256, 0, stream>>>(results, n_items, e_out, evals_out);
    return cudaGetLastError();
}

}  // namespace ud
