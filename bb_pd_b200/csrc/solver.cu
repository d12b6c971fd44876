// Fused solver: the whole BB_PD time loop in one persistent cooperative kernel.
//
// Layout in HBM (built at bbpd_create, on the device for the input and Morton
// node orders and on the host for the tiled order):
//   nodes   SoA float64 (x of all nodes, then y, then z), in input order or
//           Morton order; one flags byte per node (held / prescribed DOFs). The
//           FP32 form adds the displacement split into FP32 high and low parts
//           (16 + 8 bytes per node).
//   bonds   every undirected bond is stored twice, once in the list of each
//           end node ("directed entries"). Lists keep bond order and are laid
//           out as 32-node slices (SELL-32) in groups of 4: entries 4g..4g+3
//           of the node in lane l of slice s sit contiguously at
//           slice_ptr[s] + 4 (32 g + l), so one vector load gives a lane 4
//           entries of a stream and a warp reads 32 such groups contiguously.
//           Per entry, read every step:
//             colw  u32  neighbour index (24 bits), chunk-start bit, BONDTYPE
//             cid   u16  (u32 for irregular inputs) index into a dictionary of
//                        the distinct (L0, VCF, BONDSTIFFNESS) triples (5 872 on
//                        the 1.28M-node beam; the table stays in L1/L2)
//             st    u8   fail / softening flag / "damaged" (BSF != 0) bits
//           and, only for damaged entries, BSF (float64). Optional per-entry
//           critical stretch (float64) when the law takes per-bond sc.
//
// One time step (a launch runs any number of steps):
//   phase A  warps take 32-node slices from a shared counter; each lane walks
//            its node's entries a group of 4 at a time (the next group's
//            streams load while the current group's neighbour gathers are in
//            flight), computes stretch, law, damage and bond force, and sums the
//            forces in the reference's OpenMP order (chunk partials in bond
//            order, added in chunk order).
//            Both copies of a bond see bit-identical stretch (the squared
//            components do not depend on direction), so both copies of the
//            damage state evolve identically: no atomics, no cross-warp traffic.
//            Euler-Cromer integrates the node right there (positions
//            double-buffered); ADR writes the node's Rayleigh-quotient terms
//            reduced over the warp (one partial per slice).
//   ADR      the slice partials enter a fixed 32-ary tree whose groups are
//            folded by the warp that completes them, the root giving the
//            damping coefficient cn; barrier; phase B applies the central-
//            difference half-step update; barrier.
// Grid barriers spin with a time limit; on expiry they set an error flag and
// the kernel returns early (status BBPD_ERR_TIMEOUT), never hanging.
#include "bbpd_internal.h"
#include "divide.cuh"
#include "physics.cuh"
#include "staging.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace bbpd;

namespace {

constexpr uint32_t COL_MASK = 0x00FFFFFFu;
constexpr uint32_t F_CHUNK = 1u << 24;   // first entry of a new OpenMP chunk in this list
constexpr int BT_SHIFT = 25;             // bits 25-26: BONDTYPE
constexpr uint8_t ST_BROKEN = 1;         // fail == 0
constexpr uint8_t ST_SOFT = 2;           // flagBondSoftening == 1
constexpr uint8_t ST_DAMAGED = 4;        // BSF != +0.0 (BSF stored in bsf[])
constexpr uint8_t ST_MASK = 7;           // the three state bits
constexpr int LST_BT_SHIFT = 3;          // lattice form: bits 3-4 of the state byte hold BONDTYPE
constexpr uint8_t LST_ABSENT = 0x80;     // lattice form: no bond in this slot
constexpr int64_t MAX_NODES = (int64_t)1 << 24;

constexpr int ERR_TIMEOUT = 1;
constexpr int ERR_NONFINITE = 2;

constexpr int kBlock = 256;
#ifndef BBPD_MIN_BLOCKS
#define BBPD_MIN_BLOCKS 2       // resident blocks per SM, FP64 kernels
#endif
#ifndef BBPD_MIN_BLOCKS_F32
#define BBPD_MIN_BLOCKS_F32 2   // resident blocks per SM, FP32 dictionary-vector kernels
#endif
constexpr int kMaxLevels = 8;     // 32-ary reduction tree over the slices
constexpr int64_t kReactCap = 4096;  // per-step reactions kept from one launch

// Tiled kernel: nodes per tile, and the local neighbour word of an entry
// (12-bit index into the tile's staged nodes, chunk-start bit, BONDTYPE).
constexpr int kTile = 512;
constexpr int kTileSlices = kTile / 32;
constexpr uint32_t TJ_MASK = 0x0FFFu;
constexpr uint32_t TF_CHUNK = 1u << 12;
constexpr int TBT_SHIFT = 13;
constexpr int kTileCapMax = 4096;        // staged nodes per tile (12-bit local index)
constexpr int kDictCache = 1024;         // dictionary entries kept in shared memory

// Kernel precision variants. The FP32 form runs as kP32X when the bond vectors
// compress into its dictionary (16-bit ids); otherwise the solver runs the
// FP64 kernel, which is faster there than FP32 arithmetic on FP64 differences.
// kP32D (FP64 differences, FP32 force) is the FP32 form's general path.
constexpr int kP64 = 0, kP32D = 1, kP32X = 2;

// Entry k of the list of lane `lane` in the slice whose entries start at sbase:
// each lane's entries come in groups of 4 contiguous slots, lanes interleaved
// group by group, so a lane reads 4 entries of a stream with one vector load
// and a warp reads 32 such groups contiguously.
__host__ __device__ __forceinline__ int64_t entry_pos(int64_t sbase, int64_t k, int lane)
{
    return sbase + ((k >> 2) * 32 + lane) * 4 + (k & 3);
}

// One dictionary entry: the bond constants in FP64 and RN(1/L0) for the
// shared-divisor division. rl0 is set to -1 when a constant is not finite or
// L0 lies outside [2^-100, 2^100]: entries using it take the general path.
struct DictEntry {
    double l0, rl0, vcf, bs;
};

struct Dev {
    int64_t n_nodes, n_slices;
    const int64_t *slice_ptr;
    const int32_t *deg;
    const int32_t *slice_len;        // longest list of each slice
    const uint32_t *colw;            // global-gather kernels: neighbour word per entry
    const uint16_t *jw;              // tiled kernel: local neighbour word per entry
    int64_t n_tiles;
    const int64_t *halo_ptr;         // halo of tile t: halo[halo_ptr[t] .. halo_ptr[t+1])
    const uint32_t *halo;            // device ids of the nodes outside a tile that it reads
    int tile_cap;                    // largest tile + halo (staged nodes per block)
    int ncache;                      // dictionary entries cached in shared memory
    const void *cid;
    uint8_t *st;
    double *bsf;
    const DictEntry *dict;
    const float4 *dictx;             // FP32 form, 2 per entry: (xi_x, xi_y, xi_z, L0), (k32, |xi|^2-L0^2, regular, 0)
    float4 *urh0, *urh1;             // FP32 form: per node (uh_x, uh_y, uh_z, ul_x), ping-pong like positions
    float2 *url0, *url1;             // FP32 form: per node (ul_y, ul_z); uh + ul is the FP32 split of u
    const double *s0e, *s1e, *sce;   // per-entry law stretches or null
    double s0q;                      // FP32 fast path's s0: the scalar s0, or the least per-entry s0
                                     // (entries above it take the general path, which reads their own)
    double *smax;                    // damage-energy tracking: largest stretch of each concrete entry past s0, or null
    const double *X;
    double *xb0, *xb1;               // positions: step n reads xb[(n-1)&1], writes xb[n&1]
    double4 *xa0, *xa1;              // the same positions as (x, y, z, 0) per node: one 32-byte load per neighbour gather
    double *u, *v, *a;
    double *F0, *F1;                 // F of step n lives in F[n&1]
    const double *mass, *rho;
    const uint8_t *nflag;            // bit d: held (constrained or prescribed); bit 3+d: prescribed
    double2 *tree;                   // partial sums (cn1, cn2) of every tree level
    double *tree3;                   // partial sums of the reaction, same tree
    double *react;                   // reaction of step `it` of the last launch at [it]
    int64_t react_cap;               // entries of react[]
    int n_probe;                     // DOFs recorded every step (0: none)
    int64_t probe_node[8];           // device node of probe k
    int probe_dof[8];                // 0 x, 1 y, 2 z
    double *probe_hist;              // displacement of probe k at step it of the launch: [it * n_probe + k]
    int n_pen;                       // contact cylinders (0: none)
    double pen_cx[4], pen_r[4], pen_inc[4];
    int pen_react[4];                // 1: force counts toward the reaction
    int64_t pen_off[5];              // family of cylinder p: contact entries [pen_off[p], pen_off[p+1])
    const int32_t *cidx;             // per node: its contact entry, or -1
    // lattice form (lstep_kernel): bond slot f * n_nodes + lo holds the bond
    // between node lo and node lo + offset f of the forward stencil
    int n_sigma;                     // chain positions, a multiple of 4 (the table travels as an LTab)
    const uint64_t *lcpos;           // per node: chain positions opening an OpenMP chunk, 8 bits each, 0xFF none
    int lnx, lny, lnz;               // lattice nodes per axis
    int lty, ltz, lhalo;             // tile rows per y and z (a tile is 32 nodes long in x), stencil reach
    int lsx, lsy, lsz;               // staged box per tile: (32 + 2 reach) x (lty + 2 reach) x (ltz + 2 reach)
    int64_t ltiles[3];               // tiles per axis
    double *cforce;                  // per contact entry: z force of the step, two buffers by step parity
    double *pen_cz;                  // centre z of every cylinder, two buffers by step parity ([2][4])
    int64_t n_contact;
    int law;                         // BBPD_LAW_* (read by the batch kernel)
    int prec;                        // kernel precision variant (read by the batch kernel)
    unsigned *tcnt;                  // arrival counters of the groups of levels >= 2
    int64_t lvl_cnt[kMaxLevels];     // values at level L (level 1: one per slice)
    int64_t lvl_off[kMaxLevels];     // offset of level L in tree[]
    int64_t cnt_off[kMaxLevels];     // offset in tcnt[] of the groups forming level L
    int n_levels;
    double *scal;                    // [0] = cn
    unsigned *bar;                   // [0] arrivals, [1] generation
    unsigned long long *work;        // slice counter of phase A, zeroed before each launch
    unsigned *sticky;                // bit 0: a coordinate left the range of the fast division
    int *err;
    LawScalars P;
    double V, dt, damping;
    int amplitude;
    double rate, applied_final;
    int64_t n_time_steps;
    double guard;
    unsigned long long timeout_ns;
};

// Lattice form: the chain table, passed by value with the launch so that its
// entries are warp-uniform constant-bank reads.
constexpr int kMaxSigma = 128;
struct LTab {
    int4 e[kMaxSigma];   // (partner offset in the staged box, slot row base, lower-node offset, 0)
};

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ double prescribed_value(const Dev &d, int64_t n)
{
    if (d.amplitude == BBPD_AMP_SMOOTHSTEP) {
        // smoothstepdata(n, 1, nTimeSteps, 0, appliedDisplacement), smoothstepdata.m:40-42
        double v0 = 0.0, v1 = d.applied_final;
        double xi = ((double)n - 1.0) / ((double)d.n_time_steps - 1.0);
        return v0 + (v1 - v0) * ((xi * xi) * xi) * (10 - 15 * xi + 6 * (xi * xi));
    }
    return d.rate * (double)n;
}

// Wait until *word differs from `old`, at most timeout_ns. Gives up early when
// another block already reported a timeout in *err. On expiry sets
// ERR_TIMEOUT in *err and returns false; never waits without a limit.
__device__ bool bounded_wait_change(volatile unsigned *word, unsigned old, int *err,
                                    unsigned long long timeout_ns)
{
    const unsigned long long t0 = globaltimer();
    while (*word == old) {
        if (*(volatile int *)err & ERR_TIMEOUT) return false;
        if (globaltimer() - t0 > timeout_ns) {
            atomicOr(err, ERR_TIMEOUT);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// Clamp of calculatedampingcoefficient.m:90-112 applied to the two sums.
__device__ __forceinline__ double cn_from_sums(double cn1, double cn2)
{
    double cn;
    if (cn2 != 0) {
        if ((cn1 / cn2) > 0) cn = 2 * sqrt(cn1 / cn2);
        else cn = 0;
    } else {
        cn = 0;
    }
    if (cn > 2) cn = 1.9;
    return cn;
}

// The Rayleigh-quotient sums of one slice enter the fixed 32-ary tree: the
// warp stores its partial, and the warp that completes a group of 32 partials
// (arrival counter, fence) folds the group with the xor butterfly and carries
// the result one level up, until the root yields cn. The order of every
// addition depends on slice indices only, never on timing or launch shape.
// A third sum, the reaction (internal force summed over the prescribed DOFs),
// rides the same tree; the root stores it for step `it` of the launch.
__device__ void tree_publish(const Dev &d, int64_t sl, int lane, double c1, double c2, double c3,
                             int64_t it)
{
    int L = 1;
    int64_t idx = sl;
    for (;;) {
        if (lane == 0) {
            d.tree[d.lvl_off[L] + idx] = make_double2(c1, c2);
            d.tree3[d.lvl_off[L] + idx] = c3;
        }
        const int64_t cnt = d.lvl_cnt[L];
        if (cnt == 1) {   // root
            if (lane == 0) {
                d.scal[0] = cn_from_sums(c1, c2);
                d.scal[1] = c1;
                d.scal[2] = c2;
                d.scal[3] = c3;
                if (it < d.react_cap) d.react[it] = c3;
            }
            return;
        }
        const int64_t g = idx >> 5;
        const int gsize = (int)min((int64_t)32, cnt - g * 32);
        __threadfence();
        unsigned old = 0;
        if (lane == 0) old = atomicAdd(&d.tcnt[d.cnt_off[L + 1] + g], 1u);
        old = __shfl_sync(0xffffffffu, old, 0);
        if ((int)old != gsize - 1) return;   // another warp completes this group
        if (lane == 0) d.tcnt[d.cnt_off[L + 1] + g] = 0u;
        __threadfence();
        double2 v = make_double2(0.0, 0.0);
        double v3 = 0.0;
        if (lane < gsize) {
            v = __ldcg(&d.tree[d.lvl_off[L] + g * 32 + lane]);
            v3 = __ldcg(&d.tree3[d.lvl_off[L] + g * 32 + lane]);
        }
        c1 = v.x;
        c2 = v.y;
        c3 = v3;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            c1 = c1 + __shfl_xor_sync(0xffffffffu, c1, off);
            c2 = c2 + __shfl_xor_sync(0xffffffffu, c2, off);
            c3 = c3 + __shfl_xor_sync(0xffffffffu, c3, off);
        }
        L++;
        idx = g;
    }
}

// Next value of a work counter for this warp (lane 0 takes it, all lanes
// receive it).
__device__ __forceinline__ int64_t grab_counter(unsigned long long *ctr, int lane)
{
    unsigned long long v = 0;
    if (lane == 0) v = atomicAdd(ctr, 1ull);
    return (int64_t)__shfl_sync(0xffffffffu, v, 0);
}

__device__ __forceinline__ int64_t grab_slice(const Dev &d, int lane) { return grab_counter(d.work, lane); }

// Grid-wide barrier with a time limit on bar[0] (arrivals) and bar[1]
// (generation). False on timeout (ERR_TIMEOUT set in *err).
__device__ bool grid_barrier_raw(unsigned *bar, int *err, unsigned long long timeout_ns)
{
    __shared__ int s_last, s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = bar + 1;
        unsigned g = *gen;
        __threadfence();
        unsigned prev = atomicAdd(bar, 1u);
        s_last = (prev == gridDim.x - 1);
        s_ok = 1;
        if (!s_last) s_ok = bounded_wait_change(gen, g, err, timeout_ns) ? 1 : 0;
    }
    __syncthreads();
    if (s_last) {
        if (threadIdx.x == 0) {
            bar[0] = 0;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        }
    }
    __threadfence();
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ bool grid_barrier(const Dev &d) { return grid_barrier_raw(d.bar, d.err, d.timeout_ns); }

// L2 prefetch of one line: no register is written, so a warp can keep many
// groups of its streams in flight ahead of the loads that consume them.
__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

#ifndef BBPD_PREFETCH_GROUPS
#define BBPD_PREFETCH_GROUPS 8   // groups of 4 entries prefetched ahead of the loads
#endif
constexpr int kPrefetch = BBPD_PREFETCH_GROUPS;

__device__ __forceinline__ DictEntry ldg_dict(const DictEntry *t, uint32_t c)
{
    // the table is read-only for the whole launch: one 256-bit read-only load
    DictEntry e;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(e.l0), "=d"(e.rl0), "=d"(e.vcf), "=d"(e.bs)
        : "l"(t + c));
    return e;
}

// FP32 form: the two float4 of dictionary entry c in one 256-bit read-only load.
__device__ __forceinline__ void ldg_dictx(const float4 *t, uint32_t c, float4 &A, float4 &B)
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(A.x), "=f"(A.y), "=f"(A.z), "=f"(A.w), "=f"(B.x), "=f"(B.y), "=f"(B.z), "=f"(B.w)
        : "l"(t + 2 * (size_t)c));
}

// Per-entry data, fetched before the arithmetic of the entry. sc is the
// per-entry critical stretch when the law takes one (SCE), else the scalar.
struct Fetch {
    uint32_t w;
    uint32_t sv;
    uint32_t c;
    double xj, yj, zj, sc;
    DictEntry g;
};

// The streams of one group of 4 entries of one lane.
template <class CID> struct Group;
template <> struct Group<uint16_t> {
    uint4 w;
    uint2 c;
    uint32_t s;
    __device__ __forceinline__ uint32_t cid(int q) const
    {
        const uint32_t h = (q < 2) ? c.x : c.y;
        return (q & 1) ? (h >> 16) : (h & 0xFFFFu);
    }
};
template <> struct Group<uint32_t> {
    uint4 w;
    uint4 c;
    uint32_t s;
    __device__ __forceinline__ uint32_t cid(int q) const
    {
        return q == 0 ? c.x : q == 1 ? c.y : q == 2 ? c.z : c.w;
    }
};

template <class CID>
__device__ __forceinline__ uint32_t group_w(const Group<CID> &G, int q)
{
    return q == 0 ? G.w.x : q == 1 ? G.w.y : q == 2 ? G.w.z : G.w.w;
}

// Streams are read once per step: evict-first, so the node arrays keep L2.
template <class CID>
__device__ __forceinline__ void load_group(const Dev &d, int64_t e0, Group<CID> &G)
{
    G.w = __ldcs(reinterpret_cast<const uint4 *>(d.colw + e0));
    if constexpr (sizeof(CID) == 2)
        G.c = __ldcs(reinterpret_cast<const uint2 *>(reinterpret_cast<const uint16_t *>(d.cid) + e0));
    else
        G.c = __ldcs(reinterpret_cast<const uint4 *>(reinterpret_cast<const uint32_t *>(d.cid) + e0));
    G.s = __ldcs(reinterpret_cast<const uint32_t *>(d.st + e0));
}

// Per-entry critical stretch: SCE 1 reads the per-entry stream, 0 takes the
// scalar, 2 decides from the descriptor at run time (batch members).
template <int SCE>
__device__ __forceinline__ bool has_sce(const Dev &d)
{
    return SCE == 1 || (SCE == 2 && d.sce != nullptr);
}

template <class CID, int SCE>
__device__ __forceinline__ void prefetch_group(const Dev &d, int64_t e0)
{
    prefetch_l2(d.colw + e0);
    prefetch_l2(reinterpret_cast<const CID *>(d.cid) + e0);
    prefetch_l2(d.st + e0);
    if (has_sce<SCE>(d)) prefetch_l2(d.sce + e0);
}

// First groups of slice sl, prefetched before its turn (within the slice's
// padded length).
template <class CID, int SCE>
__device__ __forceinline__ void prefetch_slice_head(const Dev &d, int64_t sl, int lane)
{
    if (sl >= d.n_slices) return;
    const int64_t sb = d.slice_ptr[sl];
    const int ng = min(kPrefetch, d.slice_len[sl] >> 2);
    for (int g = 0; g < ng; g++) prefetch_group<CID, SCE>(d, entry_pos(sb, 4 * g, lane));
}

// Critical stretch whose crossing breaks a bond under the brittle law
// (calculatebondfailureMex.c:36-38).
__device__ __forceinline__ double linear_crit(const LawScalars &P, int bt, double sc)
{
    return (bt == 1) ? 3 * sc : (bt == 2 ? P.sc_steel : sc);
}

// True when the law cannot change the state of an intact, undamaged bond
// (state byte 0) at stretch s; NaN stretch counts as quiet.
template <int LAW>
__device__ __forceinline__ bool law_quiet(const LawScalars &P, int bt, double s, double s0,
                                          double sc)
{
    if (LAW == BBPD_LAW_LINEAR) return !(s > linear_crit(P, bt, sc));
    return !(bt == 0 && s > s0);
}

// One entry in full generality: law, damage state written back when it
// changes, bond force with the NaN guards of calculatebondforcesMex.c. Kept
// out of line: intact bonds whose law is quiet never come here.
#ifdef BBPD_GENERAL_OUTLINE
#define BBPD_GENERAL_ATTR __noinline__
#else
#define BBPD_GENERAL_ATTR __forceinline__
#endif
template <int LAW, int PREC>
__device__ BBPD_GENERAL_ATTR double3 entry_general(const Dev &d, int64_t e, uint32_t w, uint32_t sv,
                                              DictEntry g, double scb, double xi, double yi,
                                              double zi, double xj, double yj, double zj)
{
    const LawScalars &P = d.P;
    const int bt = (w >> BT_SHIFT) & 3;
    const double s0b = d.s0e ? __ldg(d.s0e + e) : P.s0;
    const double s1b = d.s1e ? __ldg(d.s1e + e) : P.s1;
    double dX, dY, dZ, L, s;
    float sf = 0.f, Lf = 0.f;
    bool exact = true;
    if (PREC == kP64) {
        bond_kinematics(xi, yi, zi, xj, yj, zj, g.l0, dX, dY, dZ, L, s);
    } else {
        dX = xj - xi; dY = yj - yi; dZ = zj - zi;
        const double L2 = dX * dX + dY * dY + dZ * dZ;
        const double diff = L2 - g.l0 * g.l0;
        const float l0f = (float)g.l0;
        Lf = sqrtf((float)L2);
        sf = (float)diff / (l0f * (Lf + l0f));
        const double crit = (LAW == BBPD_LAW_LINEAR) ? linear_crit(P, bt, scb) : scb;
        exact = fabs((double)sf - crit) < d.guard;
        if (exact) {
            L = sqrt(L2);
            s = (L - g.l0) / g.l0;
        } else {
            s = (double)sf;
            L = (double)Lf;
        }
    }
    // damage-energy tracking: every step in which a concrete bond's stretch
    // exceeds s0 comes here (the fast path requires s <= s0)
    if (d.smax && bt == 0 && s > s0b && s > d.smax[e]) d.smax[e] = s;
    // law and damage (calculatebsf*.m / calculatebondfailureMex.c)
    const double B0 = (sv & ST_DAMAGED) ? d.bsf[e] : 0.0;
    double B = B0;
    bool soft = (sv & ST_SOFT) != 0;
    double failv = (sv & ST_BROKEN) ? 0.0 : 1.0;
    const bool concrete = (bt == 0);
    if (LAW == BBPD_LAW_TRILINEAR) {
        law_trilinear(s, s0b, s1b, scb, P, d.s0e != nullptr || d.s1e != nullptr, concrete, B, soft);
    } else if (LAW == BBPD_LAW_BILINEAR) {
        law_bilinear(s, s0b, scb, concrete, B, soft);
    } else if (LAW == BBPD_LAW_EXPONENTIAL) {
        law_exponential(s, s0b, scb, P, concrete, B, soft);
    } else {
        law_linear(s, scb, P, bt, failv);
    }
    const bool dmg = __double_as_longlong(B) != 0;
    // bits above the three state bits (the lattice form's BONDTYPE) are kept
    const uint32_t stn = (soft ? ST_SOFT : 0u) | (failv == 0.0 ? ST_BROKEN : 0u) | (dmg ? ST_DAMAGED : 0u) |
                         (sv & ~(uint32_t)ST_MASK);
    if (stn != sv) d.st[e] = (uint8_t)stn;
    if (__double_as_longlong(B) != __double_as_longlong(B0)) d.bsf[e] = B;
    // bond force (calculatebondforcesMex.c:34-40)
    double3 f;
    if (PREC == kP64 || exact) {
        const double t = bond_force_scalar(failv, g.bs, B, s, 0.0, d.V, g.vcf);
        f.x = bond_force_component(t, dX, L);
        f.y = bond_force_component(t, dY, L);
        f.z = bond_force_component(t, dZ, L);
    } else {
        const float tf = (float)(failv * g.bs * (1 - B)) * sf * (float)(d.V * g.vcf);
        const float r = tf / Lf;
        float gx = r * (float)dX, gy = r * (float)dY, gz = r * (float)dZ;
        if (gx != gx) gx = 0.f;
        if (gy != gy) gy = 0.f;
        if (gz != gz) gz = 0.f;
        f.x = (double)gx; f.y = (double)gy; f.z = (double)gz;
    }
    return f;
}

// Force of one entry (FP64). The common case, an intact and undamaged bond whose law
// stays quiet, is computed inline: with fail = 1 and BSF = 0 the reference
// product fail*BS*(1-BSF)*s*V*VCF rounds exactly like ((BS*s)*V)*VCF, and with
// 0 < L < inf and a regular dictionary entry (rl0 > 0) no NaN can arise.
template <int LAW, int PREC>
__device__ __forceinline__ double3 entry_force(const Dev &d, int64_t e, const Fetch &f, bool safe,
                                               double xi, double yi, double zi)
{
    const int bt = (f.w >> BT_SHIFT) & 3;
    const double s0b = d.s0e ? __ldg(d.s0e + e) : d.P.s0;
    double3 r;
    {
        // calculatedeformedlengthMex.c:37-43 with its division by L0 and the
        // three of calculatebondforcesMex.c:34-36 by L done as correctly
        // rounded quotients with shared reciprocals (divide.cuh): bit-identical
        // to IEEE division whenever `safe` holds.
        const double dX = f.xj - xi, dY = f.yj - yi, dZ = f.zj - zi;
        const double L = sqrt(dX * dX + dY * dY + dZ * dZ);
        const double s = quot_rn(L - f.g.l0, f.g.l0, f.g.rl0);
        bool okr;
        const double rL = recip_rn(L, okr);
        if (safe && okr && f.sv == 0 && f.g.rl0 > 0 && L > 0 &&
            law_quiet<LAW>(d.P, bt, s, s0b, f.sc)) {
            const double t = ((f.g.bs * s) * d.V) * f.g.vcf;
            r.x = t * quot_rn(dX, L, rL);
            r.y = t * quot_rn(dY, L, rL);
            r.z = t * quot_rn(dZ, L, rL);
            return r;
        }
    }
    return entry_general<LAW, PREC>(d, e, f.w, f.sv, f.g, f.sc, xi, yi, zi, f.xj, f.yj, f.zj);
}

// A node's (x, y, z) from its 32-byte position record in one 256-bit load.
__device__ __forceinline__ void load_pos(const double4 *p, double &x, double &y, double &z)
{
    double w;
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(x), "=d"(y), "=d"(z), "=d"(w) : "l"(p));
    (void)w;
}

// Forces of the 32 nodes of one slice (FP64 form).
// Lane `lane` owns node sl*32+lane and walks its entries in bond order, a group
// of 4 at a time: the next group's streams load while the current group's 12
// coordinate gathers are issued together and its entries computed. Returns the
// node's force summed in the reference's order.
template <int LAW, int PREC, class CID, int SCE>
__device__ __forceinline__ void slice_forces(const Dev &d, int64_t sl, int lane, bool safe,
                                             const double *xs, const double4 *xa, double &tx, double &ty,
                                             double &tz)
{
    const int64_t nN = d.n_nodes;
    const int64_t i = sl * 32 + lane;
    const int dg = (i < nN) ? d.deg[i] : 0;
    const int64_t sb = d.slice_ptr[sl];
    const double *x0 = xs, *x1 = xs + nN, *x2 = xs + 2 * nN;

    double xi = 0, yi = 0, zi = 0;
    if (i < nN) { xi = x0[i]; yi = x1[i]; zi = x2[i]; }
    tx = 0.0; ty = 0.0; tz = 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0;

    const int ng = (dg + 3) >> 2;
    Group<CID> Gc, Gn;
    int64_t e0 = entry_pos(sb, 0, lane);
    if (ng > 0) load_group<CID>(d, e0, Gc);
    for (int g = 0; g < ng; g++, e0 += 128) {
        if (g + kPrefetch < ng) prefetch_group<CID, SCE>(d, e0 + 128 * kPrefetch);
        if (g + 1 < ng) load_group<CID>(d, e0 + 128, Gn);
        const int nq = min(4, dg - 4 * g);
        // Slots past the lane's list are layout padding (all streams zero):
        // they name node 0 and dictionary entry 0, so every slot gathers a
        // valid record and the pass below needs no per-slot selects.
        double xj[4], yj[4], zj[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t j = group_w(Gc, q) & COL_MASK;
            load_pos(xa + j, xj[q], yj[q], zj[q]);
        }
        // pass 1: the fast path of all entries of the group, without
        // branches, so that the four dependency chains interleave
        double fx[4], fy[4], fz[4];
        unsigned slow = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const bool valid = q < nq;
            const uint32_t w = group_w(Gc, q), c = Gc.cid(q), sv = (Gc.s >> (8 * q)) & 0xFFu;
            const DictEntry g = ldg_dict(d.dict, c);
            const double scv = has_sce<SCE>(d) ? __ldcs(d.sce + e0 + q) : d.P.sc;
            const double s0b = d.s0e ? __ldg(d.s0e + e0 + q) : d.P.s0;
            const int bt = (w >> BT_SHIFT) & 3;
            const double dX = xj[q] - xi, dY = yj[q] - yi, dZ = zj[q] - zi;
            const double L = sqrt(dX * dX + dY * dY + dZ * dZ);
            const double s = quot_rn(L - g.l0, g.l0, g.rl0);
            bool okr;
            const double rL = recip_rn(L, okr);
            const bool fast = safe && okr && sv == 0 && g.rl0 > 0 && L > 0 && law_quiet<LAW>(d.P, bt, s, s0b, scv);
            const double t = ((g.bs * s) * d.V) * g.vcf;
            fx[q] = t * quot_rn(dX, L, rL);
            fy[q] = t * quot_rn(dY, L, rL);
            fz[q] = t * quot_rn(dZ, L, rL);
            if (valid && !fast) slow |= 1u << q;
        }
        // pass 2: the sum in the reference's order. A full group with no
        // general entry and no chunk start (nearly every group) adds its four
        // forces straight; otherwise each entry is taken in turn.
        const uint32_t chunk = (Gc.w.x | Gc.w.y | Gc.w.z | Gc.w.w) & F_CHUNK;
        if (nq == 4 && (slow | chunk) == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) { ax = ax + fx[q]; ay = ay + fy[q]; az = az + fz[q]; }
            Gc = Gn;
            continue;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (q < nq) {
                const uint32_t w = group_w(Gc, q);
                double3 r = make_double3(fx[q], fy[q], fz[q]);
                if (slow & (1u << q)) {
                    const uint32_t j = w & COL_MASK;
                    const double scv = has_sce<SCE>(d) ? __ldcs(d.sce + e0 + q) : d.P.sc;
                    r = entry_general<LAW, PREC>(d, e0 + q, w, (Gc.s >> (8 * q)) & 0xFFu,
                                                 ldg_dict(d.dict, Gc.cid(q)), scv, xi, yi, zi, x0[j], x1[j], x2[j]);
                }
                if (w & F_CHUNK) {  // partial of the previous OpenMP thread is complete
                    tx = tx + ax; ty = ty + ay; tz = tz + az;
                    ax = 0.0; ay = 0.0; az = 0.0;
                }
                ax = ax + r.x; ay = ay + r.y; az = az + r.z;
            }
        }
        Gc = Gn;
    }
    tx = tx + ax; ty = ty + ay; tz = tz + az;
}

// General path of the FP32 dictionary-vector form: FP64 positions of both
// nodes, then the general entry in difference form.
template <int LAW>
__device__ __forceinline__ double3 entry_general_x(const Dev &d, int64_t e, uint32_t w, uint32_t sv,
                                                uint32_t c, double scd, int64_t i, const double *xs)
{
    const int64_t nN = d.n_nodes;
    const uint32_t j = w & COL_MASK;
    return entry_general<LAW, kP32D>(d, e, w, sv, ldg_dict(d.dict, c), scd, xs[i], xs[i + nN],
                                     xs[i + 2 * nN], xs[j], xs[j + nN], xs[j + 2 * nN]);
}

// FP32 form, dictionary bond vectors (kP32X). Lane `lane` owns node sl*32+lane.
// The deformed bond vector is e = xi + eta: xi = X_j - X_i from the dictionary
// (FP32), eta = (uh_j - uh_i) + (ul_j - ul_i) from the displacement split into
// FP32 high and low parts, stored as a 16-byte and an 8-byte array per node so
// that a warp's gathers of consecutive nodes read whole sectors (eta keeps close
// to FP64 accuracy under rigid translation), and
//   L^2 - L0^2 = eta . (2 xi + eta) + (|xi|^2 - L0^2),  s = (L^2 - L0^2) / (L0 (L + L0))
// is computed without cancellation; force = BS V VCF s e / L in FP32, summed in
// FP64 in the reference's order. Bonds whose stretch lies within the guard band
// of the critical stretch, damaged or broken bonds and bonds whose law is active
// take the general path with FP64 positions.
// PF: L2 prefetch of the streams ahead of the next group's loads. The single-
// beam kernel runs faster without it (0.72 against 0.77 ms/step on the
// 1.28M-node beam), the batch kernel with it (0.897 against 1.020 ms/step on a
// 16-beam batch).
template <int LAW, class CID, int SCE, bool PF>
__device__ __forceinline__ void slice_forces_x(const Dev &d, int64_t sl, int lane, const double *xs,
                                               const float4 *urh, const float2 *url, double &tx,
                                               double &ty, double &tz)
{
    const int64_t nN = d.n_nodes;
    const int64_t i = sl * 32 + lane;
    const int dg = (i < nN) ? d.deg[i] : 0;
    const int64_t sb = d.slice_ptr[sl];

    float4 ui = make_float4(0.f, 0.f, 0.f, 0.f);
    float2 li = make_float2(0.f, 0.f);
    if (i < nN) { ui = urh[i]; li = url[i]; }
    tx = 0.0; ty = 0.0; tz = 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0;
    const float s0f = (float)d.s0q, guardf = (float)d.guard, scf0 = (float)d.P.sc;
    const float steelf = (float)d.P.sc_steel;

    const int ng = (dg + 3) >> 2;
    Group<CID> Gc, Gn;
    int64_t e0 = entry_pos(sb, 0, lane);
    if (ng > 0) load_group<CID>(d, e0, Gc);
    for (int g = 0; g < ng; g++, e0 += 128) {
        if (PF && g + kPrefetch < ng) prefetch_group<CID, SCE>(d, e0 + 128 * kPrefetch);
        if (g + 1 < ng) load_group<CID>(d, e0 + 128, Gn);
        const int nq = min(4, dg - 4 * g);
        // padding slots name node 0 and dictionary entry 0 (see slice_forces)
        float4 uj[4];
        float2 lj[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t j = group_w(Gc, q) & COL_MASK;
            uj[q] = urh[j];
            lj[q] = url[j];
        }
        // pass 1: the fast path of all entries of the group, without branches,
        // so that the four dependency chains interleave
        float fxq[4], fyq[4], fzq[4];
        unsigned slow = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const bool valid = q < nq;
            const int64_t e = e0 + q;
            const uint32_t w = group_w(Gc, q), c = Gc.cid(q), sv = (Gc.s >> (8 * q)) & 0xFFu;
            const int bt = (w >> BT_SHIFT) & 3;
            float4 A, Bv;
            ldg_dictx(d.dictx, c, A, Bv);
            const float etx = (uj[q].x - ui.x) + (uj[q].w - ui.w);
            const float ety = (uj[q].y - ui.y) + (lj[q].x - li.x);
            const float etz = (uj[q].z - ui.z) + (lj[q].y - li.y);
            const float ex = A.x + etx, ey = A.y + ety, ez = A.z + etz;
            const float L2 = __fmaf_rn(ez, ez, __fmaf_rn(ey, ey, __fmul_rn(ex, ex)));
            const float rL = rsqrtf(L2);
            const float L = L2 * rL;
            const float num = __fmaf_rn(etz, A.z + ez, __fmaf_rn(ety, A.y + ey, __fmaf_rn(etx, A.x + ex, Bv.y)));
            const float sf = __fdividef(num, A.w * (L + A.w));
            // Fast iff the law is quiet and sf is outside the guard band round
            // the critical stretch (band edges rounded outwards); a NaN
            // stretch (zero, infinite or NaN length) fails every comparison.
            const float scf = has_sce<SCE>(d) ? (float)__ldcs(d.sce + e) : scf0;
            bool fast;
            if (LAW == BBPD_LAW_LINEAR) {
                const float critf = (bt == 0) ? scf : (bt == 1 ? 3.f * scf : steelf);
                fast = sf <= __fsub_rd(critf, guardf);
            } else {
                const float top = (bt == 0) ? s0f : INFINITY;
                fast = sf <= top && (sf <= __fsub_rd(scf, guardf) || sf >= __fadd_ru(scf, guardf));
            }
            fast = fast && sv == 0 && Bv.z != 0.f;
            const float qf = Bv.x * sf * rL;
            fxq[q] = qf * ex;
            fyq[q] = qf * ey;
            fzq[q] = qf * ez;
            if (valid && !fast) slow |= 1u << q;
        }
        // pass 2: the sum in the reference's order; a full group with no
        // general entry and no chunk start adds its four forces straight
        const uint32_t chunk = (Gc.w.x | Gc.w.y | Gc.w.z | Gc.w.w) & F_CHUNK;
        if (nq == 4 && (slow | chunk) == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                ax = ax + (double)fxq[q]; ay = ay + (double)fyq[q]; az = az + (double)fzq[q];
            }
            Gc = Gn;
            continue;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (q < nq) {
                const uint32_t w = group_w(Gc, q);
                double3 r;
                if (slow & (1u << q)) {
                    const double scd = has_sce<SCE>(d) ? __ldcs(d.sce + e0 + q) : d.P.sc;
                    r = entry_general_x<LAW>(d, e0 + q, w, (Gc.s >> (8 * q)) & 0xFFu, Gc.cid(q), scd, i, xs);
                } else {
                    r = make_double3((double)fxq[q], (double)fyq[q], (double)fzq[q]);
                }
                if (w & F_CHUNK) {  // partial of the previous OpenMP thread is complete
                    tx = tx + ax; ty = ty + ay; tz = tz + az;
                    ax = 0.0; ay = 0.0; az = 0.0;
                }
                ax = ax + r.x; ay = ay + r.y; az = az + r.z;
            }
        }
        Gc = Gn;
    }
    tx = tx + ax; ty = ty + ay; tz = tz + az;
}



// Coordinates for which the shared-divisor division of divide.cuh is exact:
// +0, or a magnitude in [2^-100, 2^100] (a -0 coordinate could make a -0
// numerator, whose quotient sign the fast division does not track).
__device__ __forceinline__ bool coord_out_of_range(double x)
{
    const double a = fabs(x);
    return (a != 0 || signbit(x)) && !(a >= 0x1p-100 && a <= 0x1p100);
}

// Buffers of step n: forces of this and the previous step, positions read and
// written (double-buffered), FP32 displacement split read and written, and the
// prescribed displacement of step n + 1.
struct StepBufs {
    int64_t n;
    double *Fc;
    const double *Fp, *xs;
    double *xn;
    const double4 *xas;
    double4 *xan;
    const float4 *urhs;
    const float2 *urls;
    float4 *urhn;
    float2 *urln;
    double Un1;
};

__device__ __forceinline__ StepBufs step_bufs(const Dev &d, int64_t n)
{
    StepBufs b;
    b.n = n;
    b.Fc = (n & 1) ? d.F1 : d.F0;
    b.Fp = (n & 1) ? d.F0 : d.F1;
    b.xs = ((n - 1) & 1) ? d.xb1 : d.xb0;
    b.xn = (n & 1) ? d.xb1 : d.xb0;
    b.xas = ((n - 1) & 1) ? d.xa1 : d.xa0;
    b.xan = (n & 1) ? d.xa1 : d.xa0;
    b.urhs = ((n - 1) & 1) ? d.urh1 : d.urh0;
    b.urls = ((n - 1) & 1) ? d.url1 : d.url0;
    b.urhn = (n & 1) ? d.urh1 : d.urh0;
    b.urln = (n & 1) ? d.url1 : d.url0;
    b.Un1 = prescribed_value(d, n + 1);
    return b;
}

// calculatecontactforce.m:43-82 for node i right after its integration (u,
// v, x: its displacement, velocity and position). Families are disjoint, so
// every node meets at most one cylinder and the per-node work is independent;
// the cylinder's centre for step n is the stored one of step n - 1 plus the
// increment, the same accumulation as the reference. The node's z force on
// the cylinder goes to cforce for the step's reaction sum.
__device__ __forceinline__ void apply_contact(const Dev &d, int64_t n, int64_t i, double u[3], double v[3],
                                              double x[3])
{
    const int k = d.cidx[i];
    if (k < 0) return;
    int p = 0;
    while (p + 1 < d.n_pen && k >= d.pen_off[p + 1]) p++;
    const double cz = d.pen_cz[((n - 1) & 1) * 4 + p] + d.pen_inc[p];
    const double cx = d.pen_cx[p], R = d.pen_r[p];
    const double dX = x[0] - cx, dZ = x[2] - cz;
    const double dist = sqrt((dX * dX) + (dZ * dZ));
    double fz = 0.0;
    if (dist < R) {
        const double ux = dX / dist, uz = dZ / dist;
        x[0] = cx + (ux * R);
        x[2] = cz + (uz * R);
        const int64_t nN = d.n_nodes;
        double un[3], vn[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            un[c] = x[c] - d.X[i + c * nN];
            vn[c] = (un[c] - u[c]) / d.dt;
        }
        fz = -1 * d.rho[i] * (vn[2] - v[2]) / d.dt * d.V;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            u[c] = un[c];
            v[c] = vn[c];
        }
    }
    d.cforce[(n & 1) * d.n_contact + k] = fz;
}

// Record the final displacement of node i for the probes on it (CMOD and
// similar per-step outputs, dynamicsolverdisplacementcontrolled.m:118).
__device__ __forceinline__ void record_probes(const Dev &d, int64_t it, int64_t i, const double u[3])
{
    if (it >= d.react_cap) return;
    for (int k = 0; k < d.n_probe; k++)
        if (d.probe_node[k] == i) d.probe_hist[it * d.n_probe + k] = u[d.probe_dof[k]];
}

// Once during step n (one thread): store the centres of step n, which nodes
// of step n + 1 read (nodes of step n read those of step n - 1).
__device__ __forceinline__ void contact_advance(const Dev &d, int64_t n)
{
    for (int p = 0; p < d.n_pen; p++)
        d.pen_cz[(n & 1) * 4 + p] = d.pen_cz[((n - 1) & 1) * 4 + p] + d.pen_inc[p];
}

// After step n (every node done; one thread): the reaction of the step, the
// forces of the flagged cylinders summed in family order
// (dynamicsolverdisplacementcontrolled.m:115 with calculatecontactforce.m:88).
__device__ __forceinline__ void contact_reaction(const Dev &d, int64_t n, int64_t it)
{
    double r = 0.0;
    bool first = true;
    const double *f = d.cforce + (n & 1) * d.n_contact;
    for (int p = 0; p < d.n_pen; p++) {
        if (!d.pen_react[p]) continue;
        double fz = 0.0;
        for (int64_t k = d.pen_off[p]; k < d.pen_off[p + 1]; k++) fz = fz + f[k];
        r = first ? fz : r + fz;
        first = false;
    }
    if (it < d.react_cap) d.react[it] = r;
}

// Euler-Cromer (timeintegrationeulercromerMex.c:33-50) on node i once its
// nodal force (tx, ty, tz) is summed.
template <int PREC>
__device__ __forceinline__ void ec_integrate_node(const Dev &d, const StepBufs &b, int64_t i, double tx,
                                                  double ty, double tz, int64_t it)
{
    const int64_t nN = d.n_nodes;
    const uint8_t fl = d.nflag[i];
    const double Fv[3] = {tx, ty, tz};
    double un[3], vn[3], xn3[3];
#pragma unroll
    for (int dof = 0; dof < 3; dof++) {
        const int64_t e = i + nN * dof;
        b.Fc[e] = Fv[dof];
        double ae = (Fv[dof] - d.damping * d.v[e]) / d.rho[i];
        if (fl & (1 << dof)) ae = 0;
        double ve = d.v[e] + (ae * d.dt);
        double ue = d.u[e] + (ve * d.dt);
        double xe = d.X[e] + ue;
        if (fl & (8 << dof)) { ue = b.Un1; xe = d.X[e] + ue; }
        if (d.a) d.a[e] = ae;
        un[dof] = ue; vn[dof] = ve; xn3[dof] = xe;
    }
    if (d.n_pen) apply_contact(d, b.n, i, un, vn, xn3);
    if (d.n_probe) record_probes(d, it, i, un);
    float uh[3], ul[3];
    bool bad = false, far = false;
#pragma unroll
    for (int dof = 0; dof < 3; dof++) {
        const int64_t e = i + nN * dof;
        d.v[e] = vn[dof]; d.u[e] = un[dof]; b.xn[e] = xn3[dof];
        uh[dof] = (float)un[dof]; ul[dof] = (float)(un[dof] - (double)uh[dof]);
        bad |= !isfinite(un[dof]) || !isfinite(vn[dof]);
        far |= coord_out_of_range(xn3[dof]);
    }
    if (PREC != kP32X) b.xan[i] = make_double4(xn3[0], xn3[1], xn3[2], 0.0);   // FP64 gathers only
    if (PREC == kP32X) {
        b.urhn[i] = make_float4(uh[0], uh[1], uh[2], ul[0]);
        b.urln[i] = make_float2(ul[1], ul[2]);
    }
    if (bad) atomicOr(d.err, ERR_NONFINITE);
    if (far) atomicOr(d.sticky, 1u);
}

// ADR: calculatedampingcoefficient.m:61-85 terms of the nodes of slice sl
// (lane's node has force tx, ty, tz) and their share of the reaction (force on
// the prescribed DOFs), folded over the slice's 32 lanes by the xor butterfly
// and entered into the tree.
__device__ __forceinline__ void adr_slice_terms(const Dev &d, const StepBufs &b, int64_t sl, int lane,
                                                double tx, double ty, double tz, int64_t it)
{
    const int64_t nN = d.n_nodes;
    const int64_t i = sl * 32 + lane;
    double c1 = 0, c2 = 0, c3 = 0;
    if (i < nN) {
        const double m = d.mass[i];
        const double Fv[3] = {tx, ty, tz};
        const uint8_t fl = d.nflag[i];
#pragma unroll
        for (int dof = 0; dof < 3; dof++)
            if (fl & (8 << dof)) c3 = c3 + Fv[dof];
#pragma unroll
        for (int dof = 0; dof < 3; dof++) {
            const int64_t e = i + nN * dof;
            const double vhp = d.v[e], ue = d.u[e];
            if (vhp != 0) c1 = c1 - ue * ue * ((Fv[dof] / m - b.Fp[e] / m) / (d.dt * vhp));
        }
#pragma unroll
        for (int dof = 0; dof < 3; dof++) {
            const double ue = d.u[i + nN * dof];
            c2 = c2 + ue * ue;
        }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        c1 = c1 + __shfl_xor_sync(0xffffffffu, c1, off);
        c2 = c2 + __shfl_xor_sync(0xffffffffu, c2, off);
        c3 = c3 + __shfl_xor_sync(0xffffffffu, c3, off);
    }
    tree_publish(d, sl, lane, c1, c2, c3, it);
}

// Work on one slice after its nodal forces (tx, ty, tz of lane's node) are
// summed: Euler-Cromer integrates the node; ADR stores F, forms the node's
// Rayleigh-quotient terms, folds them over the slice and enters the tree.
template <int SCHEME, int PREC>
__device__ __forceinline__ void finish_slice(const Dev &d, const StepBufs &b, int64_t sl, int lane,
                                             double tx, double ty, double tz, int64_t it)
{
    const int64_t nN = d.n_nodes;
    const int64_t i = sl * 32 + lane;
    const bool valid = i < nN;
    if (SCHEME == BBPD_SCHEME_EULERCROMER) {
        if (valid) ec_integrate_node<PREC>(d, b, i, tx, ty, tz, it);
    } else {
        if (valid) { b.Fc[i] = tx; b.Fc[i + nN] = ty; b.Fc[i + 2 * nN] = tz; }
        adr_slice_terms(d, b, sl, lane, tx, ty, tz, it);
    }
}

// ADR phase B (timeintegrationADR.m:53-80) on the nodes of slice sb.
template <int PREC>
__device__ __forceinline__ void adr_update_slice(const Dev &d, const StepBufs &b, int64_t sb, int lane,
                                                 int64_t it)
{
    const int64_t nN = d.n_nodes;
    const double cn = __ldcg(&d.scal[0]);
    {
        const int64_t i = sb * 32 + lane;
        if (i >= nN) return;
        const uint8_t fl = d.nflag[i];
        const double minv = 1.0 / d.mass[i];
        double un[3], vn[3], xn3[3];
#pragma unroll
        for (int dof = 0; dof < 3; dof++) {
            const int64_t e = i + nN * dof;
            const double F = b.Fc[e];
            double vh;
            if (b.n == 1) vh = 0.5 * d.dt * minv * F;
            else vh = (((2 - cn * d.dt) * d.v[e]) + (2 * d.dt * minv * F)) / (2 + cn * d.dt);
            double ue = d.u[e] + (d.dt * vh);
            if (fl & (1 << dof)) { ue = 0; vh = 0; }
            if (fl & (8 << dof)) { ue = b.Un1; vh = 0; }
            un[dof] = ue; vn[dof] = vh; xn3[dof] = d.X[e] + ue;
        }
        if (d.n_pen) apply_contact(d, b.n, i, un, vn, xn3);
        if (d.n_probe) record_probes(d, it, i, un);
        float uh[3], ul[3];
        bool bad = false, far = false;
#pragma unroll
        for (int dof = 0; dof < 3; dof++) {
            const int64_t e = i + nN * dof;
            d.v[e] = vn[dof]; d.u[e] = un[dof]; b.xn[e] = xn3[dof];
            uh[dof] = (float)un[dof]; ul[dof] = (float)(un[dof] - (double)uh[dof]);
            bad |= !isfinite(un[dof]) || !isfinite(vn[dof]);
            far |= coord_out_of_range(xn3[dof]);
        }
        if (PREC != kP32X) b.xan[i] = make_double4(xn3[0], xn3[1], xn3[2], 0.0);   // FP64 gathers only
        if (PREC == kP32X) {
            b.urhn[i] = make_float4(uh[0], uh[1], uh[2], ul[0]);
            b.urln[i] = make_float2(ul[1], ul[2]);
        }
        if (bad) atomicOr(d.err, ERR_NONFINITE);
        if (far) atomicOr(d.sticky, 1u);
    }
}

// ADR phase B on slices gwarp, gwarp + nwarps, ...
template <int PREC>
__device__ __forceinline__ void adr_update(const Dev &d, const StepBufs &b, int lane, int64_t gwarp,
                                           int64_t nwarps, int64_t it)
{
    for (int64_t sb = gwarp; sb < d.n_slices; sb += nwarps) adr_update_slice<PREC>(d, b, sb, lane, it);
}

// Global-gather kernel: neighbour data read from HBM/L2 per entry. Used for
// inputs whose tiles do not fit shared memory, and for input or plain Morton
// node order.
template <int LAW, int SCHEME, int PREC, class CID, bool SCE>
__global__ void __launch_bounds__(kBlock, PREC == kP32X ? BBPD_MIN_BLOCKS_F32 : BBPD_MIN_BLOCKS) step_kernel(Dev d, int64_t step0, int64_t nsteps)
{
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nsl = d.n_slices;

    for (int64_t it = 0; it < nsteps; it++) {
        const StepBufs b = step_bufs(d, step0 + it);
        const bool safe = (*(volatile unsigned *)d.sticky & 1u) == 0;
        if (d.n_pen && blockIdx.x == 0 && threadIdx.x == 0) contact_advance(d, b.n);

        // ---- phase A: bond forces (+ Euler-Cromer / ADR terms) ----
        // Warps take slices from a shared counter, so warps that finish early
        // take more. Each warp stops at its first grab past the last slice,
        // so a step uses exactly nsl + nwarps counter values and the base of
        // step `it` of this launch is it * (nsl + nwarps). Results depend on
        // slice indices only, not on which warp computes a slice.
        const int64_t base = it * (nsl + nwarps);
        int64_t sl = grab_slice(d, lane) - base;
        if (PREC != kP32X) prefetch_slice_head<CID, SCE>(d, sl, lane);   // FP32: see slice_forces_x
        while (sl < nsl) {
            const int64_t sl_next = grab_slice(d, lane) - base;
            if (PREC != kP32X) prefetch_slice_head<CID, SCE>(d, sl_next, lane);
            double tx, ty, tz;
            if (PREC == kP32X) slice_forces_x<LAW, CID, SCE, false>(d, sl, lane, b.xs, b.urhs, b.urls, tx, ty, tz);
            else slice_forces<LAW, PREC, CID, SCE>(d, sl, lane, safe, b.xs, b.xas, tx, ty, tz);
            finish_slice<SCHEME, PREC>(d, b, sl, lane, tx, ty, tz, it);
            sl = sl_next;
        }
        if (SCHEME == BBPD_SCHEME_ADR) {
            if (!grid_barrier(d)) return;
            adr_update<PREC>(d, b, lane, gwarp, nwarps, it);
        }
        if (!grid_barrier(d)) return;
        if (d.n_pen && blockIdx.x == 0 && threadIdx.x == 0) contact_reaction(d, b.n, it);
    }
}

// ---------------------------------------------------------------- tiled kernel
//
// Nodes in Morton order are cut into tiles of kTile consecutive nodes (16
// slices; an 8 x 8 x 8 brick on a regular lattice). For every tile the host
// lists the nodes outside it that its entries reference (its halo); entries
// name their neighbour by a 12-bit index into [tile nodes, halo nodes]. A block
// takes a tile, stages the positions (FP64 form) or the displacement split
// (FP32 form) of the tile and its halo into shared memory with independent
// loads, then its warps take the tile's slices and read every neighbour from
// shared memory. The most used dictionary entries stay in shared memory for the
// whole launch.

// Streams of one group of 4 entries: local neighbour words, dictionary ids, states.
struct TGroup {
    uint2 j, c;
    uint32_t s;
    __device__ __forceinline__ uint32_t jw(int q) const
    {
        const uint32_t h = (q < 2) ? j.x : j.y;
        return (q & 1) ? (h >> 16) : (h & 0xFFFFu);
    }
    __device__ __forceinline__ uint32_t cid(int q) const
    {
        const uint32_t h = (q < 2) ? c.x : c.y;
        return (q & 1) ? (h >> 16) : (h & 0xFFFFu);
    }
};

template <bool SCE>
__device__ __forceinline__ void prefetch_tgroup(const Dev &d, int64_t e0)
{
    prefetch_l2(d.jw + e0);
    prefetch_l2(reinterpret_cast<const uint16_t *>(d.cid) + e0);
    prefetch_l2(d.st + e0);
    if (SCE) prefetch_l2(d.sce + e0);
}

template <bool SCE>
__device__ __forceinline__ void prefetch_tslice_head(const Dev &d, int64_t sl, int lane)
{
    const int64_t sb = d.slice_ptr[sl];
    const int ng = min(kPrefetch, d.slice_len[sl] >> 2);
    for (int g = 0; g < ng; g++) prefetch_tgroup<SCE>(d, entry_pos(sb, 4 * g, lane));
}

__device__ __forceinline__ void load_tgroup(const Dev &d, int64_t e0, TGroup &G)
{
    G.j = __ldcs(reinterpret_cast<const uint2 *>(d.jw + e0));
    G.c = __ldcs(reinterpret_cast<const uint2 *>(reinterpret_cast<const uint16_t *>(d.cid) + e0));
    G.s = __ldcs(reinterpret_cast<const uint32_t *>(d.st + e0));
}

// Bond-type bits of a local neighbour word, placed where entry_force and
// entry_general expect them.
__device__ __forceinline__ uint32_t tword(uint32_t jw)
{
    return ((jw >> TBT_SHIFT) & 3u) << BT_SHIFT;
}

// FP64 form: forces of the 32 nodes of slice sl, lane's node at local index li.
template <int LAW, bool SCE>
__device__ __forceinline__ void tslice_forces(const Dev &d, int64_t sl, int li, int lane, bool safe,
                                              const double *sx, const double *sy, const double *sz,
                                              const DictEntry *sdict, int ncache, double &tx,
                                              double &ty, double &tz)
{
    const int64_t i = sl * 32 + lane;
    const int dg = (i < d.n_nodes) ? d.deg[i] : 0;
    const int64_t sb = d.slice_ptr[sl];
    double xi = 0, yi = 0, zi = 0;
    if (dg > 0) { xi = sx[li]; yi = sy[li]; zi = sz[li]; }
    tx = 0.0; ty = 0.0; tz = 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0;
    const int ng = (dg + 3) >> 2;
    TGroup Gc, Gn;
    int64_t e0 = entry_pos(sb, 0, lane);
    if (ng > 0) load_tgroup(d, e0, Gc);
    for (int g = 0; g < ng; g++, e0 += 128) {
        if (g + kPrefetch < ng) prefetch_tgroup<SCE>(d, e0 + 128 * kPrefetch);
        if (g + 1 < ng) load_tgroup(d, e0 + 128, Gn);
        const int nq = min(4, dg - 4 * g);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (q < nq) {
                const uint32_t jw = Gc.jw(q), jl = jw & TJ_MASK;
                Fetch f;
                f.w = tword(jw);
                f.c = Gc.cid(q);
                f.sv = (Gc.s >> (8 * q)) & 0xFFu;
                f.sc = SCE ? __ldcs(d.sce + e0 + q) : d.P.sc;
                f.xj = sx[jl]; f.yj = sy[jl]; f.zj = sz[jl];
                f.g = ((int)f.c < ncache) ? sdict[f.c] : ldg_dict(d.dict, f.c);
                const double3 r = entry_force<LAW, kP64>(d, e0 + q, f, safe, xi, yi, zi);
                if (jw & TF_CHUNK) {  // partial of the previous OpenMP thread is complete
                    tx = tx + ax; ty = ty + ay; tz = tz + az;
                    ax = 0.0; ay = 0.0; az = 0.0;
                }
                ax = ax + r.x; ay = ay + r.y; az = az + r.z;
            }
        }
        Gc = Gn;
    }
    tx = tx + ax; ty = ty + ay; tz = tz + az;
}

// FP32 dictionary-vector form on staged displacement splits (see slice_forces_x
// for the arithmetic). Neighbours outside the fast path read FP64 positions
// from HBM through the tile's halo list.
template <int LAW, bool SCE>
__device__ __forceinline__ void tslice_forces_x(const Dev &d, int64_t sl, int li, int lane,
                                                int64_t n0, int nt, int64_t hp,
                                                const float4 *suh, const float2 *sul,
                                                const float4 *sdx, int ncache, const double *xs,
                                                double &tx, double &ty, double &tz)
{
    const int64_t nN = d.n_nodes;
    const int64_t i = sl * 32 + lane;
    const int dg = (i < nN) ? d.deg[i] : 0;
    const int64_t sb = d.slice_ptr[sl];
    float4 ui = make_float4(0.f, 0.f, 0.f, 0.f);
    float2 vi = make_float2(0.f, 0.f);
    if (dg > 0) { ui = suh[li]; vi = sul[li]; }
    tx = 0.0; ty = 0.0; tz = 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0;
    const float s0f = (float)d.s0q, guardf = (float)d.guard;
    const int ng = (dg + 3) >> 2;
    TGroup Gc, Gn;
    int64_t e0 = entry_pos(sb, 0, lane);
    if (ng > 0) load_tgroup(d, e0, Gc);
    for (int g = 0; g < ng; g++, e0 += 128) {
        if (g + kPrefetch < ng) prefetch_tgroup<SCE>(d, e0 + 128 * kPrefetch);
        if (g + 1 < ng) load_tgroup(d, e0 + 128, Gn);
        const int nq = min(4, dg - 4 * g);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (q < nq) {
                const int64_t e = e0 + q;
                const uint32_t jw = Gc.jw(q), jl = jw & TJ_MASK, c = Gc.cid(q);
                const uint32_t sv = (Gc.s >> (8 * q)) & 0xFFu, w = tword(jw);
                const double scd = SCE ? __ldcs(d.sce + e) : d.P.sc;
                const int bt = (w >> BT_SHIFT) & 3;
                const bool hit = (int)c < ncache;
                const float4 A = hit ? sdx[2 * c] : __ldg(&d.dictx[2 * c]);
                const float4 Bv = hit ? sdx[2 * c + 1] : __ldg(&d.dictx[2 * c + 1]);
                const float4 uj = suh[jl];
                const float2 vj = sul[jl];
                const float etx = (uj.x - ui.x) + (uj.w - ui.w);
                const float ety = (uj.y - ui.y) + (vj.x - vi.x);
                const float etz = (uj.z - ui.z) + (vj.y - vi.y);
                const float ex = A.x + etx, ey = A.y + ety, ez = A.z + etz;
                const float L2 = __fmaf_rn(ez, ez, __fmaf_rn(ey, ey, __fmul_rn(ex, ex)));
                const float rL = rsqrtf(L2);
                const float L = L2 * rL;
                const float num = __fmaf_rn(etz, A.z + ez, __fmaf_rn(ety, A.y + ey, __fmaf_rn(etx, A.x + ex, Bv.y)));
                const float sf = __fdividef(num, A.w * (L + A.w));
                const float crit = (float)((LAW == BBPD_LAW_LINEAR) ? linear_crit(d.P, bt, scd) : scd);
                const float s0b = s0f;   // least per-entry s0: entries above it take the general path
                const bool quiet = (LAW == BBPD_LAW_LINEAR) ? !(sf > crit) : !(bt == 0 && sf > s0b);
                double3 r;
                if (sv == 0 && Bv.z != 0.f && L2 > 0.f && L2 < INFINITY && !(fabsf(sf - crit) < guardf) && quiet) {
                    const float qf = Bv.x * sf * rL;
                    r.x = (double)(qf * ex);
                    r.y = (double)(qf * ey);
                    r.z = (double)(qf * ez);
                } else {
                    const int64_t gj = ((int)jl < nt) ? n0 + jl : (int64_t)d.halo[hp + jl - nt];
                    r = entry_general<LAW, kP32D>(d, e, w, sv, ldg_dict(d.dict, c), scd, xs[i], xs[i + nN],
                                                  xs[i + 2 * nN], xs[gj], xs[gj + nN], xs[gj + 2 * nN]);
                }
                if (jw & TF_CHUNK) {  // partial of the previous OpenMP thread is complete
                    tx = tx + ax; ty = ty + ay; tz = tz + az;
                    ax = 0.0; ay = 0.0; az = 0.0;
                }
                ax = ax + r.x; ay = ay + r.y; az = az + r.z;
            }
        }
        Gc = Gn;
    }
    tx = tx + ax; ty = ty + ay; tz = tz + az;
}

// Dynamic shared memory of the tiled kernel: the dictionary cache (ncache
// entries of 32 bytes) followed by the staged node data of one tile (tile_cap
// nodes of 24 bytes: x, y, z in FP64, or the FP32 split as float4 + float2).
template <int LAW, int SCHEME, int PREC, bool SCE>
__global__ void __launch_bounds__(kBlock, 2) tstep_kernel(Dev d, int64_t step0, int64_t nsteps)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int64_t s_tile;
    __shared__ int s_next;
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nN = d.n_nodes, ntiles = d.n_tiles;
    const int ncache = d.ncache, cap = d.tile_cap;

    DictEntry *sdict = reinterpret_cast<DictEntry *>(smem);
    float4 *sdx = reinterpret_cast<float4 *>(smem);
    unsigned char *stage = smem + (size_t)32 * ncache;
    double *sx = reinterpret_cast<double *>(stage), *sy = sx + cap, *sz = sy + cap;
    float4 *suh = reinterpret_cast<float4 *>(stage);
    float2 *sul = reinterpret_cast<float2 *>(suh + cap);

    for (int c = threadIdx.x; c < ncache; c += blockDim.x) {
        if (PREC == kP32X) {
            sdx[2 * c] = __ldg(&d.dictx[2 * c]);
            sdx[2 * c + 1] = __ldg(&d.dictx[2 * c + 1]);
        } else {
            sdict[c] = ldg_dict(d.dict, c);
        }
    }

    for (int64_t it = 0; it < nsteps; it++) {
        const StepBufs b = step_bufs(d, step0 + it);
        const bool safe = (*(volatile unsigned *)d.sticky & 1u) == 0;
        if (d.n_pen && blockIdx.x == 0 && threadIdx.x == 0) contact_advance(d, b.n);
        // Blocks take tiles from a shared counter; each block stops at its
        // first grab past the last tile, so a step uses exactly
        // ntiles + gridDim.x counter values.
        const int64_t base = it * (ntiles + gridDim.x);
        for (;;) {
            if (threadIdx.x == 0) {
                s_tile = (int64_t)atomicAdd(d.work, 1ull) - base;
                s_next = 0;
            }
            __syncthreads();
            const int64_t tile = s_tile;
            if (tile >= ntiles) break;
            const int64_t n0 = tile * kTile;
            const int nt = (int)min((int64_t)kTile, nN - n0);
            const int64_t hp = d.halo_ptr[tile];
            const int nloc = nt + (int)(d.halo_ptr[tile + 1] - hp);
            {
                const int w = threadIdx.x >> 5;
                if (w * 32 < nt) prefetch_tslice_head<SCE>(d, tile * kTileSlices + w, lane);
            }
            for (int l = threadIdx.x; l < nloc; l += blockDim.x) {
                const int64_t g = (l < nt) ? n0 + l : (int64_t)d.halo[hp + l - nt];
                if (PREC == kP32X) {
                    suh[l] = b.urhs[g];
                    sul[l] = b.urls[g];
                } else {
                    sx[l] = b.xs[g];
                    sy[l] = b.xs[g + nN];
                    sz[l] = b.xs[g + 2 * nN];
                }
            }
            __syncthreads();
            const int nslt = (nt + 31) / 32;
            const int nwb = blockDim.x >> 5;
            for (;;) {
                int k = 0;
                if (lane == 0) k = atomicAdd(&s_next, 1);
                k = __shfl_sync(0xffffffffu, k, 0);
                if (k >= nslt) break;
                const int64_t sl = tile * kTileSlices + k;
                if (k + nwb < nslt) prefetch_tslice_head<SCE>(d, sl + nwb, lane);
                double tx, ty, tz;
                if (PREC == kP32X)
                    tslice_forces_x<LAW, SCE>(d, sl, k * 32 + lane, lane, n0, nt, hp, suh, sul, sdx, ncache,
                                              b.xs, tx, ty, tz);
                else
                    tslice_forces<LAW, SCE>(d, sl, k * 32 + lane, lane, safe, sx, sy, sz, sdict, ncache,
                                            tx, ty, tz);
                finish_slice<SCHEME, PREC>(d, b, sl, lane, tx, ty, tz, it);
            }
            __syncthreads();
        }
        if (SCHEME == BBPD_SCHEME_ADR) {
            if (!grid_barrier(d)) return;
            adr_update<PREC>(d, b, lane, gwarp, nwarps, it);
        }
        if (!grid_barrier(d)) return;
        if (d.n_pen && blockIdx.x == 0 && threadIdx.x == 0) contact_reaction(d, b.n, it);
    }
}

// ---------------------------------------------------------------- lattice kernel
//
// Lattice form, for a regular lattice of nodes in x-fastest order (the order
// of buildmaterialpointcoordinates.m:38-56) whose bond list gives every node
// its bonds in one common order of stencil offsets (a bond list ordered by
// its first node, each node's family in one order: what buildbonddata.m
// builds on such a lattice). Neighbours are then addressed by the stencil, not
// stored: each bond has one slot, slot = f * nN + lo for the bond from node lo
// to node lo + f (f a forward stencil offset), holding a state byte (fail /
// softening / damaged bits, BONDTYPE, "absent" for offsets that leave the
// lattice or bonds that are not in the list) and a dictionary id, read by both
// end nodes. Both ends compute bit-identical stretch and the same law update
// from the same state, so either may store the new state; the update is
// idempotent (max, or, and), so the other end computes the same force whether
// it reads the state before or after the store.
//
// A block takes a tile of 32 x lty x ltz nodes, stages the positions of the
// tile and of the stencil's reach around it in shared memory, and each warp
// walks one row of 32 nodes, one lane per node. Lanes read their partners at
// a fixed offset of their own staged position, so the 32 lanes read 32
// consecutive doubles (no bank conflicts), and the slots of one chain position
// are consecutive too (coalesced). Each node sums its entries in its bond-list
// order, with the OpenMP chunk partials of calculatenodalforcesopenmpMex.c.
// Euler-Cromer integrates each node in the tile; ADR stores the forces, and
// the Rayleigh-quotient sums run over 32-node slices after a grid barrier, in
// the same tree as the other kernels.

// Forces of lane's node n (own: its index in the staged box). Every chain
// position is computed without branches, absent ones included: their slot
// holds dictionary id 0 and their staged partner a finite position (or 0
// outside the lattice), and only present entries enter the sum.
template <int LAW, bool SCE>
__device__ __forceinline__ void lattice_forces(const Dev &d, int n, bool valid, int own, bool safe,
                                               const double *sx, const double *sy, const double *sz,
                                               const LTab &tab, const DictEntry *sdict, int ncache,
                                               double &tx, double &ty, double &tz)
{
    const uint16_t *cids = reinterpret_cast<const uint16_t *>(d.cid);
    const uint8_t *sts = d.st;
    const double xi = sx[own], yi = sy[own], zi = sz[own];
    uint64_t cp = valid ? __ldg(d.lcpos + n) : ~0ull;
    int nextc = (int)(cp & 0xFFu);
    tx = 0.0; ty = 0.0; tz = 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0;
    const int ng = d.n_sigma >> 2;
    // state bytes and dictionary ids of one group of 4 chain positions; slot
    // rows are padded by the stencil's reach on both sides, so every
    // n + lower-node offset addresses a slot of its row (padding is absent)
    uint32_t Sc[4], Cc[4], Sn[4], Cn[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int slot = tab.e[q].y + n + tab.e[q].z;
        Sc[q] = __ldcs(sts + slot);
        Cc[q] = __ldcs(cids + slot);
    }
    for (int g = 0; g < ng; g++) {
        if (g + 1 < ng) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int slot = tab.e[4 * g + 4 + q].y + n + tab.e[4 * g + 4 + q].z;
                Sn[q] = __ldcs(sts + slot);
                Cn[q] = __ldcs(cids + slot);
            }
        }
        double fx[4], fy[4], fz[4];
        unsigned slow = 0, pres = 0;
        // pass 1: the fast path of the group's four entries, without branches
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int4 t = tab.e[4 * g + q];
            const uint32_t sv = Sc[q];
            const int p = own + t.x;
            const double dX = sx[p] - xi, dY = sy[p] - yi, dZ = sz[p] - zi;
            const uint32_t c = Cc[q];
            DictEntry gd;
            if ((int)c < ncache) gd = sdict[c];
            else gd = ldg_dict(d.dict, c);
            const double scv = SCE ? __ldcs(d.sce + (t.y + n + t.z)) : d.P.sc;
            const int bt = (sv >> LST_BT_SHIFT) & 3;
            const double L = sqrt(dX * dX + dY * dY + dZ * dZ);
            const double s = quot_rn(L - gd.l0, gd.l0, gd.rl0);
            bool okr;
            const double rL = recip_rn(L, okr);
            const bool fast = safe && okr && (sv & ST_MASK) == 0 && gd.rl0 > 0 && L > 0 &&
                              law_quiet<LAW>(d.P, bt, s, d.P.s0, scv);
            const double tt = ((gd.bs * s) * d.V) * gd.vcf;
            fx[q] = tt * quot_rn(dX, L, rL);
            fy[q] = tt * quot_rn(dY, L, rL);
            fz[q] = tt * quot_rn(dZ, L, rL);
            const bool present = valid && !(sv & LST_ABSENT);
            pres |= (present ? 1u : 0u) << q;
            slow |= (present && !fast ? 1u : 0u) << q;
        }
        // pass 2: the rare general entries, and the sum in the reference's order
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (pres & (1u << q)) {
                const int sig = 4 * g + q;
                double3 r = make_double3(fx[q], fy[q], fz[q]);
                if (slow & (1u << q)) {
                    const int4 t = tab.e[sig];
                    const int slot = t.y + n + t.z;
                    const uint32_t sv = Sc[q];
                    const int p = own + t.x;
                    const double scv = SCE ? __ldcs(d.sce + slot) : d.P.sc;
                    const uint32_t w = ((sv >> LST_BT_SHIFT) & 3u) << BT_SHIFT;
                    r = entry_general<LAW, kP64>(d, slot, w, sv, ldg_dict(d.dict, Cc[q]), scv, xi, yi, zi,
                                                 sx[p], sy[p], sz[p]);
                }
                if (sig == nextc) {   // partial of the previous OpenMP thread is complete
                    tx = tx + ax; ty = ty + ay; tz = tz + az;
                    ax = 0.0; ay = 0.0; az = 0.0;
                    cp >>= 8;
                    nextc = (int)(cp & 0xFFu);
                }
                ax = ax + r.x; ay = ay + r.y; az = az + r.z;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) { Sc[q] = Sn[q]; Cc[q] = Cn[q]; }
    }
    tx = tx + ax; ty = ty + ay; tz = tz + az;
}

// Dynamic shared memory: the dictionary cache (ncache entries of 32 bytes)
// and the staged positions of one tile (x, y, z arrays over the lsx * lsy *
// lsz box).
template <int LAW, int SCHEME, bool SCE>
__global__ void __launch_bounds__(kBlock, 2) lstep_kernel(Dev d, int64_t step0, int64_t nsteps, LTab tab)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int64_t s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nN = d.n_nodes, nsl = d.n_slices;
    const int ncache = d.ncache;
    const int sxn = d.lsx, syn = d.lsy, szn = d.lsz, H = d.lhalo;
    const int box = sxn * syn * szn;
    const int64_t ntx = d.ltiles[0], nty = d.ltiles[1], ntiles = d.ltiles[0] * d.ltiles[1] * d.ltiles[2];

    DictEntry *sdict = reinterpret_cast<DictEntry *>(smem);
    double *sx = reinterpret_cast<double *>(smem + (size_t)32 * ncache), *sy = sx + box, *sz = sy + box;

    for (int c = threadIdx.x; c < ncache; c += blockDim.x) sdict[c] = ldg_dict(d.dict, c);

    // this warp's row in a tile
    const int wy = warp % d.lty, wz = warp / d.lty;
    const bool wrow = warp < d.lty * d.ltz;
    const int own = (lane + H) + sxn * ((wy + H) + syn * (wz + H));

    for (int64_t it = 0; it < nsteps; it++) {
        const StepBufs b = step_bufs(d, step0 + it);
        const bool safe = (*(volatile unsigned *)d.sticky & 1u) == 0;
        if (d.n_pen && blockIdx.x == 0 && threadIdx.x == 0) contact_advance(d, b.n);
        // tiles from a shared counter; each block stops at its first grab past
        // the last tile, so a step uses exactly ntiles + gridDim.x values
        const int64_t base = it * (ntiles + gridDim.x);
        for (;;) {
            __syncthreads();   // the previous tile's positions are no longer read
            if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(d.work, 1ull) - base;
            __syncthreads();
            const int64_t tile = s_tile;
            if (tile >= ntiles) break;
            const int64_t tz0 = tile / (ntx * nty), rem = tile - tz0 * ntx * nty;
            const int64_t ty0 = rem / ntx, tx0 = rem - ty0 * ntx;
            const int x0 = (int)tx0 * 32, y0 = (int)ty0 * d.lty, z0 = (int)tz0 * d.ltz;
            // stage the tile and its reach; points outside the lattice hold 0
            for (int l = threadIdx.x; l < box; l += blockDim.x) {
                const int bz = l / (sxn * syn), r2 = l - bz * sxn * syn;
                const int by = r2 / sxn, bx = r2 - by * sxn;
                const int gx = x0 - H + bx, gy = y0 - H + by, gz = z0 - H + bz;
                double px = 0.0, py = 0.0, pz = 0.0;
                if (gx >= 0 && gx < d.lnx && gy >= 0 && gy < d.lny && gz >= 0 && gz < d.lnz) {
                    const int64_t g = gx + (int64_t)d.lnx * (gy + (int64_t)d.lny * gz);
                    px = b.xs[g]; py = b.xs[g + nN]; pz = b.xs[g + 2 * nN];
                }
                sx[l] = px; sy[l] = py; sz[l] = pz;
            }
            __syncthreads();
            if (wrow) {
                const int gx = x0 + lane, gy = y0 + wy, gz = z0 + wz;
                const bool valid = gx < d.lnx && gy < d.lny && gz < d.lnz;
                const int n = valid ? gx + d.lnx * (gy + d.lny * gz) : 0;
                double tx, ty, tz;
                lattice_forces<LAW, SCE>(d, n, valid, own, safe, sx, sy, sz, tab, sdict, ncache, tx, ty, tz);
                if (valid) {
                    if (SCHEME == BBPD_SCHEME_EULERCROMER) {
                        ec_integrate_node<kP64>(d, b, n, tx, ty, tz, it);
                    } else {
                        b.Fc[n] = tx; b.Fc[n + nN] = ty; b.Fc[n + 2 * nN] = tz;
                    }
                }
            }
        }
        if (SCHEME == BBPD_SCHEME_ADR) {
            if (!grid_barrier(d)) return;
            // Rayleigh-quotient terms over 32-node slices, in the tree order
            // of the other kernels
            for (int64_t sl = gwarp; sl < nsl; sl += nwarps) {
                const int64_t i = sl * 32 + lane;
                double fx = 0, fy = 0, fz = 0;
                if (i < nN) { fx = b.Fc[i]; fy = b.Fc[i + nN]; fz = b.Fc[i + 2 * nN]; }
                adr_slice_terms(d, b, sl, lane, fx, fy, fz, it);
            }
            if (!grid_barrier(d)) return;
            adr_update<kP64>(d, b, lane, gwarp, nwarps, it);
        }
        if (!grid_barrier(d)) return;
        if (d.n_pen && blockIdx.x == 0 && threadIdx.x == 0) contact_reaction(d, b.n, it);
    }
}

// ---------------------------------------------------------------- batch kernel
//
// Many solver states ("members") of any sizes stepped together: the members
// of one class (same law and kernel variant) share one persistent launch, in
// which phase A takes slices from one counter over the concatenation of all
// members' slices (prefix[m] = first global slice of member m), so the SMs
// stay busy however uneven the members are; every member keeps its own step
// number, ADR tree, damping coefficient and reaction history, and its
// arithmetic is that of a launch of its own.
struct BatchCtl {
    const Dev *members;        // device copies of the members' descriptors
    const int64_t *prefix;     // S + 1 entries
    int64_t *mstep;            // next step of each member; advanced at the end of a launch
    int S;
    int grab;                  // consecutive slices per counter grab
    int64_t total;             // prefix[S]
    unsigned *bar;
    unsigned long long *work;
    int *err;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ int member_of(const BatchCtl &B, int64_t w)
{
    int lo = 0, hi = B.S;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&B.prefix[mid]) <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Copy member m's descriptor into this warp's shared slot (when it holds
// another member). Reads through the slot cannot alias the state the kernel
// stores to global memory, so the compiler keeps descriptor fields in
// registers as it does for a kernel parameter.
__device__ __forceinline__ const Dev &warp_member(const BatchCtl &B, int m, Dev *slot, int *held, int lane)
{
    if (*held != m) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(B.members + m);
        uint32_t *dst = reinterpret_cast<uint32_t *>(slot);
        for (int k = lane; k < (int)(sizeof(Dev) / 4); k += 32) dst[k] = __ldg(src + k);
        __syncwarp();
        if (lane == 0) *held = m;
        __syncwarp();
    }
    return *slot;
}

// The members of one class (one law, one kernel precision variant, per-entry
// critical stretch or not) stepped by one persistent launch; a batch of mixed
// classes replays one such launch per class. Every instance is as
// specialised as the single-solver kernel.
template <int LAW, int PREC, bool SCE>
__global__ void __launch_bounds__(kBlock, BBPD_MIN_BLOCKS) batch_kernel(BatchCtl B, int64_t nsteps)
{
    __shared__ Dev s_dev[kBlock / 32];
    __shared__ int s_held[kBlock / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t G = B.grab;
    const int64_t ngrabs = (B.total + G - 1) / G;
    if (lane == 0) s_held[wib] = -1;
    __syncwarp();

    for (int64_t it = 0; it < nsteps; it++) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            for (int m = 0; m < B.S; m++)
                if (B.members[m].n_pen) contact_advance(B.members[m], __ldg(&B.mstep[m]) + it);
        // one failing grab per warp and step: ngrabs + nwarps values per step
        const int64_t base = it * (ngrabs + nwarps);
        int64_t gi = grab_counter(B.work, lane) - base;
        while (gi < ngrabs) {
            const int64_t gnext = grab_counter(B.work, lane) - base;
            const int64_t w1 = min(B.total, (gi + 1) * G);
            for (int64_t w = gi * G; w < w1; w++) {
                const int m = member_of(B, w);
                const Dev &d = warp_member(B, m, &s_dev[wib], &s_held[wib], lane);
                const int64_t sl = w - __ldg(&B.prefix[m]);
                const StepBufs b = step_bufs(d, __ldg(&B.mstep[m]) + it);
                const bool safe = (*(volatile unsigned *)d.sticky & 1u) == 0;
                double tx, ty, tz;
                if (PREC == kP32X) slice_forces_x<LAW, uint16_t, SCE, true>(d, sl, lane, b.xs, b.urhs, b.urls, tx, ty, tz);
                else slice_forces<LAW, PREC, uint16_t, SCE>(d, sl, lane, safe, b.xs, b.xas, tx, ty, tz);
                finish_slice<BBPD_SCHEME_ADR, PREC>(d, b, sl, lane, tx, ty, tz, it);
            }
            gi = gnext;
        }
        if (!grid_barrier_raw(B.bar, B.err, B.timeout_ns)) return;
        for (int64_t w = gwarp; w < B.total; w += nwarps) {
            const int m = member_of(B, w);
            const Dev &d = warp_member(B, m, &s_dev[wib], &s_held[wib], lane);
            const StepBufs b = step_bufs(d, __ldg(&B.mstep[m]) + it);
            adr_update_slice<PREC>(d, b, w - __ldg(&B.prefix[m]), lane, it);
        }
        if (!grid_barrier_raw(B.bar, B.err, B.timeout_ns)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0)
            for (int m = 0; m < B.S; m++)
                if (B.members[m].n_pen) contact_reaction(B.members[m], __ldg(&B.mstep[m]) + it, it);
    }
    // every block has read the step numbers of the last step (barrier above)
    if (blockIdx.x == 0)
        for (int m = threadIdx.x; m < B.S; m += blockDim.x) B.mstep[m] += nsteps;
}

// Forces and integration terms of slice sl of member d under law LAW, out of
// line: each law keeps a register allocation of its own instead of sharing one
// sized for all four.
template <int LAW, int PREC>
__device__ __noinline__ void mixed_law_slice(const Dev &d, const StepBufs &b, int64_t sl, int lane, int64_t it)
{
    const bool safe = (*(volatile unsigned *)d.sticky & 1u) == 0;
    double tx, ty, tz;
    if (PREC == kP32X) slice_forces_x<LAW, uint16_t, 2, true>(d, sl, lane, b.xs, b.urhs, b.urls, tx, ty, tz);
    else slice_forces<LAW, PREC, uint16_t, 2>(d, sl, lane, safe, b.xs, b.xas, tx, ty, tz);
    finish_slice<BBPD_SCHEME_ADR, PREC>(d, b, sl, lane, tx, ty, tz, it);
}

// Slice sl of member d with its own law (a warp-uniform switch: a slice
// belongs to one member), reading a per-entry critical stretch when the
// member has one.
template <int PREC>
__device__ __forceinline__ void mixed_slice(const Dev &d, const StepBufs &b, int64_t sl, int lane, int64_t it)
{
    switch (d.law) {
    case BBPD_LAW_LINEAR: mixed_law_slice<BBPD_LAW_LINEAR, PREC>(d, b, sl, lane, it); break;
    case BBPD_LAW_BILINEAR: mixed_law_slice<BBPD_LAW_BILINEAR, PREC>(d, b, sl, lane, it); break;
    case BBPD_LAW_TRILINEAR: mixed_law_slice<BBPD_LAW_TRILINEAR, PREC>(d, b, sl, lane, it); break;
    default: mixed_law_slice<BBPD_LAW_EXPONENTIAL, PREC>(d, b, sl, lane, it); break;
    }
}

// Every member of a batch of one kernel precision variant, whatever its law
// and whether it reads a per-entry critical stretch, in one persistent launch
// (the schedule of batch_kernel; each member's arithmetic is that of its own
// solver's kernel).
template <int PREC>
__global__ void __launch_bounds__(kBlock, BBPD_MIN_BLOCKS) batch_kernel_mixed(BatchCtl B, int64_t nsteps)
{
    __shared__ Dev s_dev[kBlock / 32];
    __shared__ int s_held[kBlock / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t G = B.grab;
    const int64_t ngrabs = (B.total + G - 1) / G;
    if (lane == 0) s_held[wib] = -1;
    __syncwarp();

    for (int64_t it = 0; it < nsteps; it++) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            for (int m = 0; m < B.S; m++)
                if (B.members[m].n_pen) contact_advance(B.members[m], __ldg(&B.mstep[m]) + it);
        const int64_t base = it * (ngrabs + nwarps);
        int64_t gi = grab_counter(B.work, lane) - base;
        while (gi < ngrabs) {
            const int64_t gnext = grab_counter(B.work, lane) - base;
            const int64_t w1 = min(B.total, (gi + 1) * G);
            for (int64_t w = gi * G; w < w1; w++) {
                const int m = member_of(B, w);
                const Dev &d = warp_member(B, m, &s_dev[wib], &s_held[wib], lane);
                const StepBufs b = step_bufs(d, __ldg(&B.mstep[m]) + it);
                mixed_slice<PREC>(d, b, w - __ldg(&B.prefix[m]), lane, it);
            }
            gi = gnext;
        }
        if (!grid_barrier_raw(B.bar, B.err, B.timeout_ns)) return;
        for (int64_t w = gwarp; w < B.total; w += nwarps) {
            const int m = member_of(B, w);
            const Dev &d = warp_member(B, m, &s_dev[wib], &s_held[wib], lane);
            const StepBufs b = step_bufs(d, __ldg(&B.mstep[m]) + it);
            adr_update_slice<PREC>(d, b, w - __ldg(&B.prefix[m]), lane, it);
        }
        if (!grid_barrier_raw(B.bar, B.err, B.timeout_ns)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0)
            for (int m = 0; m < B.S; m++)
                if (B.members[m].n_pen) contact_reaction(B.members[m], __ldg(&B.mstep[m]) + it, it);
    }
    if (blockIdx.x == 0)
        for (int m = threadIdx.x; m < B.S; m += blockDim.x) B.mstep[m] += nsteps;
}

typedef void (*batch_kernel_t)(BatchCtl, int64_t);

batch_kernel_t pick_batch_mixed(int prec)
{
    return prec == kP32X ? batch_kernel_mixed<kP32X> : batch_kernel_mixed<kP64>;
}

template <int PREC, bool SCE>
batch_kernel_t pick_batch_law(int law)
{
    switch (law) {
    case BBPD_LAW_LINEAR: return batch_kernel<BBPD_LAW_LINEAR, PREC, SCE>;
    case BBPD_LAW_BILINEAR: return batch_kernel<BBPD_LAW_BILINEAR, PREC, SCE>;
    case BBPD_LAW_TRILINEAR: return batch_kernel<BBPD_LAW_TRILINEAR, PREC, SCE>;
    default: return batch_kernel<BBPD_LAW_EXPONENTIAL, PREC, SCE>;
    }
}

batch_kernel_t pick_batch_kernel(int law, int prec, bool sce)
{
    if (prec == kP32X) return sce ? pick_batch_law<kP32X, true>(law) : pick_batch_law<kP32X, false>(law);
    return sce ? pick_batch_law<kP64, true>(law) : pick_batch_law<kP64, false>(law);
}

// Self-test of the bounded wait: one thread waits on a word that nothing
// writes, so the wait must expire and report ERR_TIMEOUT.
__global__ void wait_selftest_kernel(unsigned *word, int *err, unsigned long long timeout_ns)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) bounded_wait_change(word, 0u, err, timeout_ns);
}

// Per-bond views of the per-entry state: bond k's two copies sit at ent[k]
// and ent[nB + k] (the copies are identical, the gather reads the first).
template <class IDX>
__global__ void k_bond_gather(const IDX *__restrict__ ent, int64_t nB, const double *__restrict__ bsf,
                              const uint8_t *__restrict__ st, int field, double *out)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nB; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pos = (int64_t)ent[k];
        if (field == BBPD_FIELD_BSF) {
            out[k] = bsf[pos];
        } else {
            const uint8_t w = st[pos];
            out[k] = field == BBPD_FIELD_FLAG ? ((w & ST_SOFT) ? 1.0 : 0.0) : ((w & ST_BROKEN) ? 0.0 : 1.0);
        }
    }
}

// calculatedamageenergy.m:34-62 for every bond from the largest stretch its
// entries recorded (the energy is a non-decreasing function of the stretch, so
// this equals the reference's running maximum over steps); bonds never past s0
// have recorded 0 and get 0.
template <class IDX, class CID>
__global__ void k_bond_energy(const IDX *__restrict__ ent, int64_t nB, const double *__restrict__ smax,
                              const CID *__restrict__ cid, const DictEntry *__restrict__ dict,
                              const double *__restrict__ s0e, const double *__restrict__ sce, double s0, double sc,
                              double shape, double den, double V2, double *out)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nB; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pos = (int64_t)ent[k];
        const double s = smax[pos], a = s0e ? s0e[pos] : s0, c = sce ? sce[pos] : sc;
        const DictEntry g = dict[cid[pos]];
        double de = 0.0;
        if ((a < s) && (s <= c)) de = (((((g.bs * a) * g.l0) * (a - s)) * shape) / den) * V2;
        else if (s > c) de = (((((g.bs * a) * g.l0) * (a - c)) * shape) / den) * V2;
        out[k] = de;
    }
}

// Flag or fail bit of every bond as one byte (0/1).
template <class IDX>
__global__ void k_bond_gather_bits(const IDX *__restrict__ ent, int64_t nB, const uint8_t *__restrict__ st,
                                   int field, uint8_t *out)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nB; k += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t w = st[(int64_t)ent[k]];
        out[k] = field == BBPD_FIELD_FLAG ? ((w & ST_SOFT) ? 1 : 0) : ((w & ST_BROKEN) ? 0 : 1);
    }
}

template <class IDX>
__global__ void k_bond_scatter(const IDX *__restrict__ ent, int64_t nB, const double *__restrict__ in, int field,
                               double *bsf, uint8_t *st)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nB; k += (int64_t)gridDim.x * blockDim.x) {
        const double v = in[k];
        for (int side = 0; side < 2; side++) {
            const int64_t pos = (int64_t)ent[side * nB + k];
            uint8_t w = st[pos];
            if (field == BBPD_FIELD_BSF) {
                bsf[pos] = v;
                w = __double_as_longlong(v) != 0 ? (uint8_t)(w | ST_DAMAGED) : (uint8_t)(w & ~ST_DAMAGED);
            } else if (field == BBPD_FIELD_FLAG) {
                w = v == 1 ? (uint8_t)(w | ST_SOFT) : (uint8_t)(w & ~ST_SOFT);
            } else {
                w = v == 0 ? (uint8_t)(w | ST_BROKEN) : (uint8_t)(w & ~ST_BROKEN);
            }
            st[pos] = w;
        }
    }
}

// ---- layout build on the device (input and Morton node orders) ----
//
// Directed entry q = 2k + side of bond k sits in the list of node key[q]
// (side 0: the bond's first BONDLIST column, side 1: its second). A stable
// radix sort of the entries by node keeps every list in bond order, exactly
// as the reference's nodal loop meets the bonds; the run bounds of the sorted
// keys give each node its degree and each entry its rank in the list.

__global__ void k_iota(uint32_t *v, int64_t n)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        v[q] = (uint32_t)q;
}

// first[p] / last[p]: sorted positions bounding node p's run (both stay 0 for
// a node without bonds)
__global__ void k_run_bounds(const uint32_t *__restrict__ skey, int64_t n, uint32_t *first, uint32_t *last)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = skey[r];
        if (r == 0 || skey[r - 1] != p) first[p] = (uint32_t)r;
        if (r == n - 1 || skey[r + 1] != p) last[p] = (uint32_t)(r + 1);
    }
}

// One warp per 32-node slice: node degrees, the slice's list length (its
// longest list rounded up to whole groups of 4) and its entry count.
__global__ void k_slice_lengths(const uint32_t *__restrict__ first, const uint32_t *__restrict__ last, int64_t nN,
                                int64_t ns, int32_t *deg, int32_t *slen, int64_t *scount)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; s < ns; s += warps) {
        const int64_t p = s * 32 + lane;
        const int32_t dg = p < nN ? (int32_t)(last[p] - first[p]) : 0;
        if (p < nN) deg[p] = dg;
        const int32_t m = (__reduce_max_sync(0xffffffffu, (unsigned)dg) + 3) & ~3;
        if (lane == 0) {
            slen[s] = m;
            scount[s] = (int64_t)m * 32;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) scount[ns] = 0;
}

struct LayoutArgs {
    const uint32_t *key;      // [2 nB] node of entry q, unsorted
    const uint32_t *skey;     // sorted keys
    const uint32_t *sval;     // sorted entry ids q
    const uint32_t *first;    // [nN] first sorted position of each node
    const int64_t *sptr;      // [ns + 1] slice offsets
    const uint16_t *bcid;     // [nB] dictionary id of the forward copy; null: id = k (32-bit ids)
    const uint16_t *negid;    // FP32 form: id of the reversed bond vector, else null
    const uint8_t *bflag;     // [nB] bit 0: fail == 0, bits 1-2: BONDTYPE; or null
    const double *s0, *s1, *sc;   // per-bond law parameters or null
    int64_t nB;
    int T;                    // OpenMP chunks of the reference's bond loop
    uint32_t *colw;
    void *cid;                // u16, or u32 when bcid is null
    uint8_t *st;
    double *s0e, *s1e, *sce;
    void *ent;                // [2 nB] bond -> entry map, u32 or i64
    int ent32;
};

// Every directed entry to its slot: neighbour, BONDTYPE and chunk-start bits,
// dictionary id, fail state, optional law parameters, and the bond -> entry
// map. An entry starts an OpenMP chunk when its bond lies in another chunk
// than the previous entry of the same list.
__global__ void k_layout_scatter(LayoutArgs a)
{
    const int64_t n = 2 * a.nB;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t q = a.sval[r], p = a.skey[r];
        const int64_t k = q >> 1;
        const int side = (int)(q & 1u);
        const int64_t rank = r - (int64_t)a.first[p];
        const int64_t pos = entry_pos(a.sptr[p >> 5], rank, (int)(p & 31u));
        const uint8_t fl = a.bflag ? a.bflag[k] : (uint8_t)0;
        const bool cs = rank == 0 || omp_chunk_of(k, a.nB, a.T) != omp_chunk_of((int64_t)(a.sval[r - 1] >> 1), a.nB, a.T);
        a.colw[pos] = a.key[q ^ 1u] | ((uint32_t)(fl >> 1) << BT_SHIFT) | (cs ? F_CHUNK : 0u);
        if (a.bcid) {
            uint16_t c = a.bcid[k];
            if (side && a.negid) c = a.negid[c];
            ((uint16_t *)a.cid)[pos] = c;
        } else {
            ((uint32_t *)a.cid)[pos] = (uint32_t)k;
        }
        a.st[pos] = (fl & 1u) ? ST_BROKEN : (uint8_t)0;
        if (a.s0) a.s0e[pos] = a.s0[k];
        if (a.s1) a.s1e[pos] = a.s1[k];
        if (a.sc) a.sce[pos] = a.sc[k];
        if (a.ent32) ((uint32_t *)a.ent)[side * a.nB + k] = (uint32_t)pos;
        else ((int64_t *)a.ent)[side * a.nB + k] = pos;
    }
}

__global__ void k_fill(double *v, int64_t n, double x)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        v[q] = x;
}

// Initial node state from the staged coordinates and flags: u holds the step-1
// prescribed value U1 on prescribed DOFs and 0 elsewhere, both position
// buffers hold X + u, and the FP32 form gets the split record of u.
__global__ void k_node_init(Dev d, double U1)
{
    const int64_t nN = d.n_nodes;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nN; p += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t f = d.nflag[p];
        bool far = false;
        float uh[3], ul[3];
        double xr[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const int64_t e = p + c * nN;
            const double u = (f & (8 << c)) ? U1 : 0.0;
            const double x = d.X[e] + u;
            d.u[e] = u;
            d.xb0[e] = x;
            d.xb1[e] = x;
            xr[c] = x;
            far |= coord_out_of_range(x);
            uh[c] = (float)u;
            ul[c] = (float)(u - (double)uh[c]);
        }
        d.xa0[p] = d.xa1[p] = make_double4(xr[0], xr[1], xr[2], 0.0);
        if (d.urh0) {
            d.urh0[p] = d.urh1[p] = make_float4(uh[0], uh[1], uh[2], ul[0]);
            d.url0[p] = d.url1[p] = make_float2(ul[1], ul[2]);
        }
        if (far) atomicOr(d.sticky, 1u);
    }
}

// Position records (x, y, z, 0) from the SoA position buffer.
__global__ void k_pack_positions(const double *__restrict__ x, int64_t nN, double4 *xa)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nN; p += (int64_t)gridDim.x * blockDim.x)
        xa[p] = make_double4(x[p], x[p + nN], x[p + 2 * nN], 0.0);
}

typedef void (*kernel_t)(Dev, int64_t, int64_t);

// Instances: law x scheme x precision x dictionary-index width x per-entry
// critical stretch. Irregular inputs (32-bit dictionary indices) are served
// with the per-entry critical stretch stream in every case.
template <int LAW, int SCHEME, int PREC>
kernel_t pick_cid(bool wide, bool sce)
{
    if constexpr (PREC != kP32X) {   // the dictionary-vector form only runs with 16-bit ids
        if (wide) return step_kernel<LAW, SCHEME, PREC, uint32_t, true>;
    }
    return sce ? step_kernel<LAW, SCHEME, PREC, uint16_t, true> : step_kernel<LAW, SCHEME, PREC, uint16_t, false>;
}

template <int LAW, int SCHEME>
kernel_t pick_prec(int prec, bool wide, bool sce)
{
    if (prec == kP32X) return pick_cid<LAW, SCHEME, kP32X>(wide, sce);
    return pick_cid<LAW, SCHEME, kP64>(wide, sce);
}

template <int LAW>
kernel_t pick_scheme(int scheme, int prec, bool wide, bool sce)
{
    return scheme == BBPD_SCHEME_ADR ? pick_prec<LAW, BBPD_SCHEME_ADR>(prec, wide, sce)
                                     : pick_prec<LAW, BBPD_SCHEME_EULERCROMER>(prec, wide, sce);
}

template <int LAW, int SCHEME>
kernel_t pick_tprec(int prec, bool sce)
{
    if (prec == kP32X) return sce ? tstep_kernel<LAW, SCHEME, kP32X, true> : tstep_kernel<LAW, SCHEME, kP32X, false>;
    return sce ? tstep_kernel<LAW, SCHEME, kP64, true> : tstep_kernel<LAW, SCHEME, kP64, false>;
}

template <int LAW>
kernel_t pick_tscheme(int scheme, int prec, bool sce)
{
    return scheme == BBPD_SCHEME_ADR ? pick_tprec<LAW, BBPD_SCHEME_ADR>(prec, sce)
                                     : pick_tprec<LAW, BBPD_SCHEME_EULERCROMER>(prec, sce);
}

// Tiled kernels: 16-bit dictionary ids, FP64 or FP32 dictionary-vector form.
kernel_t pick_tkernel(int law, int scheme, int prec, bool sce)
{
    switch (law) {
    case BBPD_LAW_LINEAR: return pick_tscheme<BBPD_LAW_LINEAR>(scheme, prec, sce);
    case BBPD_LAW_BILINEAR: return pick_tscheme<BBPD_LAW_BILINEAR>(scheme, prec, sce);
    case BBPD_LAW_TRILINEAR: return pick_tscheme<BBPD_LAW_TRILINEAR>(scheme, prec, sce);
    default: return pick_tscheme<BBPD_LAW_EXPONENTIAL>(scheme, prec, sce);
    }
}

typedef void (*lkernel_t)(Dev, int64_t, int64_t, LTab);
static_assert(sizeof(Dev) + 16 + sizeof(LTab) <= 4096, "lattice kernel parameters exceed 4 KB");

template <int LAW>
lkernel_t pick_lscheme(int scheme, bool sce)
{
    if (scheme == BBPD_SCHEME_ADR) return sce ? lstep_kernel<LAW, BBPD_SCHEME_ADR, true> : lstep_kernel<LAW, BBPD_SCHEME_ADR, false>;
    return sce ? lstep_kernel<LAW, BBPD_SCHEME_EULERCROMER, true> : lstep_kernel<LAW, BBPD_SCHEME_EULERCROMER, false>;
}

// Lattice form: FP64, 16-bit dictionary ids.
lkernel_t pick_lkernel(int law, int scheme, bool sce)
{
    switch (law) {
    case BBPD_LAW_LINEAR: return pick_lscheme<BBPD_LAW_LINEAR>(scheme, sce);
    case BBPD_LAW_BILINEAR: return pick_lscheme<BBPD_LAW_BILINEAR>(scheme, sce);
    case BBPD_LAW_TRILINEAR: return pick_lscheme<BBPD_LAW_TRILINEAR>(scheme, sce);
    default: return pick_lscheme<BBPD_LAW_EXPONENTIAL>(scheme, sce);
    }
}

kernel_t pick_kernel(int law, int scheme, int prec, bool wide, bool sce)
{
    switch (law) {
    case BBPD_LAW_LINEAR: return pick_scheme<BBPD_LAW_LINEAR>(scheme, prec, wide, sce);
    case BBPD_LAW_BILINEAR: return pick_scheme<BBPD_LAW_BILINEAR>(scheme, prec, wide, sce);
    case BBPD_LAW_TRILINEAR: return pick_scheme<BBPD_LAW_TRILINEAR>(scheme, prec, wide, sce);
    default: return pick_scheme<BBPD_LAW_EXPONENTIAL>(scheme, prec, wide, sce);
    }
}

// ------------------------------------------------------------------ host side

unsigned host_threads()
{
    return std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
}

template <class F>
void host_parallel_for(int64_t n, F fn)
{
    unsigned nt = host_threads();
    if (n < 65536) nt = 1;
    std::vector<std::thread> th;
    int64_t per = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        int64_t lo = (int64_t)t * per, hi = std::min(n, lo + per);
        if (lo >= hi) break;
        th.emplace_back([=]() { for (int64_t i = lo; i < hi; i++) fn(i); });
    }
    for (auto &x : th) x.join();
}

// Run fn(t, lo, hi) on T contiguous ranges of [0, n), one thread each.
template <class F>
void host_ranges(int64_t n, int T, F fn)
{
    std::vector<std::thread> th;
    for (int t = 0; t < T; t++) {
        int64_t lo = n * t / T, hi = n * (t + 1) / T;
        th.emplace_back([=]() { fn(t, lo, hi); });
    }
    for (auto &x : th) x.join();
}

inline int chunk_of_host(int64_t k, int64_t n, int T)
{
    int64_t q = n / T, r = n % T, big = r * (q + 1);
    if (k < big) return (int)(k / (q + 1));
    return (int)(r + (k - big) / q);
}

uint64_t morton3(uint32_t a, uint32_t b, uint32_t c)
{
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffull;
        v = (v | v << 16) & 0x1f0000ff0000ffull;
        v = (v | v << 8) & 0x100f00f00f00f00full;
        v = (v | v << 4) & 0x10c30c30c30c30c3ull;
        v = (v | v << 2) & 0x1249249249249249ull;
        return v;
    };
    return spread(a) | (spread(b) << 1) | (spread(c) << 2);
}

struct KeyX {
    uint64_t a, b, c;
    uint32_t x, y, z;
    bool operator==(const KeyX &o) const { return a == o.a && b == o.b && c == o.c && x == o.x && y == o.y && z == o.z; }
    bool operator<(const KeyX &o) const
    {
        if (a != o.a) return a < o.a;
        if (b != o.b) return b < o.b;
        if (c != o.c) return c < o.c;
        if (x != o.x) return x < o.x;
        return y != o.y ? y < o.y : z < o.z;
    }
};
struct KeyXHash {
    size_t operator()(const KeyX &k) const
    {
        uint64_t h = k.a * 0x9E3779B97F4A7C15ull ^ (k.b + 0x632BE59BD9B4E019ull) * 0xBF58476D1CE4E5B9ull;
        h ^= (k.c + 0x94D049BB133111EBull) * 0xD6E8FEB86659FD93ull;
        h ^= ((uint64_t)k.x << 32 | k.y) * 0xA24BAED4963EE407ull ^ (uint64_t)k.z * 0x9FB21C651E98DF25ull;
        return (size_t)(h ^ (h >> 29));
    }
};

inline uint32_t fbits(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
}

struct Key3 {
    uint64_t a, b, c;
    bool operator==(const Key3 &o) const { return a == o.a && b == o.b && c == o.c; }
    bool operator<(const Key3 &o) const { return a != o.a ? a < o.a : (b != o.b ? b < o.b : c < o.c); }
};
struct Key3Hash {
    size_t operator()(const Key3 &k) const
    {
        uint64_t h = k.a * 0x9E3779B97F4A7C15ull ^ (k.b + 0x632BE59BD9B4E019ull) * 0xBF58476D1CE4E5B9ull;
        h ^= (k.c + 0x94D049BB133111EBull) * 0xD6E8FEB86659FD93ull;
        return (size_t)(h ^ (h >> 29));
    }
};

// Open-addressing hash map (linear probing, power-of-two capacity, at most
// half full) from a dictionary key to a 32-bit id, for the passes over every
// bond. The slot is taken from the top bits of a Fibonacci multiply of the
// key's hash, so every bit of the hash matters.
template <class K, class H>
struct FlatMap {
    static constexpr uint32_t kEmpty = 0xFFFFFFFFu;
    std::vector<K> keys;
    std::vector<uint32_t> vals;
    int bits = 0;
    size_t count = 0;
    explicit FlatMap(int b = 10) { reset(b); }
    void reset(int b)
    {
        bits = b;
        keys.assign((size_t)1 << b, K{});
        vals.assign((size_t)1 << b, kEmpty);
        count = 0;
    }
    size_t slot(const K &k) const { return (size_t)(((uint64_t)H()(k) * 0x9E3779B97F4A7C15ull) >> (64 - bits)); }
    size_t probe(const K &k) const
    {
        const size_t mask = ((size_t)1 << bits) - 1;
        size_t h = slot(k);
        while (vals[h] != kEmpty && !(keys[h] == k)) h = (h + 1) & mask;
        return h;
    }
    // the id of k, storing v for it when k is new
    uint32_t insert(const K &k, uint32_t v)
    {
        if (2 * (count + 1) > ((size_t)1 << bits)) {
            std::vector<K> ok;
            std::vector<uint32_t> ov;
            ok.swap(keys);
            ov.swap(vals);
            reset(bits + 1);
            for (size_t i = 0; i < ov.size(); i++)
                if (ov[i] != kEmpty) {
                    const size_t h = probe(ok[i]);
                    keys[h] = ok[i];
                    vals[h] = ov[i];
                    count++;
                }
        }
        const size_t h = probe(k);
        if (vals[h] == kEmpty) {
            keys[h] = k;
            vals[h] = v;
            count++;
        }
        return vals[h];
    }
    uint32_t find(const K &k) const { return vals[probe(k)]; }
    void set(const K &k, uint32_t v) { vals[probe(k)] = v; }   // k present
    template <class F>
    void for_each(F f) const
    {
        for (size_t i = 0; i < vals.size(); i++)
            if (vals[i] != kEmpty) f(keys[i], vals[i]);
    }
};

DictEntry make_entry(double l0, double vcf, double bs)
{
    DictEntry e;
    e.l0 = l0;
    e.vcf = vcf;
    e.bs = bs;
    const bool regular = std::isfinite(vcf) && std::isfinite(bs) && l0 >= 0x1p-100 && l0 <= 0x1p100;
    e.rl0 = regular ? 1.0 / l0 : -1.0;   // IEEE division: RN(1/L0); -1 marks irregular
    return e;
}

// FP32 (high, low) split of a node-major displacement array u (x of node p
// at [p], y at [p + nN], z at [p + 2 nN]) in the two per-node arrays the
// kernels gather and write after each step: h[p] = (uh_x, uh_y, uh_z, ul_x),
// l[p] = (ul_y, ul_z), uh = RN32(u), ul = RN32(u - uh).
void split_record(const double *u, int64_t nN, std::vector<float4> &h, std::vector<float2> &l)
{
    h.resize(nN);
    l.resize(nN);
    for (int64_t p = 0; p < nN; p++) {
        float hi[3], lo[3];
        for (int c = 0; c < 3; c++) {
            const double v = u[p + c * nN];
            hi[c] = (float)v;
            lo[c] = (float)(v - (double)hi[c]);
        }
        h[p] = make_float4(hi[0], hi[1], hi[2], lo[0]);
        l[p] = make_float2(lo[1], lo[2]);
    }
}

// Coordinates for which the shared-divisor division is exact: +0, or a
// magnitude in [2^-100, 2^100].
inline bool coord_safe(double x)
{
    const double a = std::fabs(x);
    return (a == 0 && !std::signbit(x)) || (a >= 0x1p-100 && a <= 0x1p100);
}

inline uint64_t bits_of(double x)
{
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
}

}  // namespace

struct bbpd_solver {
    int device = 0;
    bbpd_params prm{};
    int64_t nN = 0, nB = 0, ns = 0, ne = 0, ndict = 0;
    bool wide = false;
    int prec = kP64;                    // kernel variant (kP64 or kP32X)
    int64_t step = 1;
    double cn = 0;
    std::vector<int32_t> perm;          // device position -> input node
    std::vector<int32_t> inv;           // input node -> device position
    std::unique_ptr<int64_t[]> ent_i, ent_j;  // bond -> entry positions of its two copies (host, until uploaded)
    void *d_ent = nullptr;              // the same on the device, [ent_i | ent_j], 32-bit when they fit
    bool ent32 = false;
    Dev d{};
    std::vector<void *> allocs;
    int64_t device_bytes = 0;
    double bytes_per_step = 0;
    kernel_t kernel = nullptr;
    int grid = 0;
    bool tiled = false;                 // tiled kernel with shared-memory staging
    bool lattice = false;               // lattice form (lstep_kernel)
    LTab ltab{};                        // its chain table, a launch argument
    size_t smem = 0;                    // its dynamic shared memory per block
    bbpd_batch *batch = nullptr;        // batch this solver is a member of
    bool has_density = false;          // DENSITY given (contact needs it)
    bool cn_stale = false;              // cn on the device is newer than S->cn
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    template <class T>
    int alloc(T **p, size_t count)
    {
        size_t b = sizeof(T) * std::max<size_t>(count, 1);
        BBPD_CUDA_TRY(cudaMalloc((void **)p, b));
        allocs.push_back((void *)*p);
        device_bytes += (int64_t)b;
        return BBPD_OK;
    }
    template <class T>
    int put(T **p, const T *h, size_t count)
    {
        int rc = alloc(p, count);
        if (rc) return rc;
        if (count) BBPD_CUDA_TRY(cudaMemcpy(*p, h, sizeof(T) * count, cudaMemcpyHostToDevice));
        return BBPD_OK;
    }
    template <class T>
    int put(T **p, const std::vector<T> &h) { return put(p, h.data(), h.size()); }
    ~bbpd_solver()
    {
        for (void *p : allocs) cudaFree(p);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

#define TRY(x) do { int r_ = (x); if (r_) return r_; } while (0)

// Wait for the batch's launches and rebuild its member table before the next
// one (a member's descriptor or step changed on the host).
static int batch_member_changed(bbpd_batch *B);

// Smallest k in [0, n) with bad(k), or -1; the ranges are checked in parallel.
template <class F>
static int64_t first_bad(int64_t n, F bad)
{
    const int HT = (int)std::min<int64_t>(host_threads(), std::max<int64_t>(1, n / 65536));
    std::vector<int64_t> first(HT, -1);
    host_ranges(n, HT, [&](int t, int64_t lo, int64_t hi) {
        for (int64_t k = lo; k < hi; k++)
            if (bad(k)) {
                first[t] = k;
                return;
            }
    });
    for (int64_t f : first)
        if (f >= 0) return f;
    return -1;
}

static int validate_01(const double *a, int64_t n, const char *name)
{
    if (!a) return BBPD_OK;
    const int64_t i = first_bad(n, [&](int64_t k) { return !(a[k] == 0.0 || a[k] == 1.0); });
    if (i >= 0) return fail(BBPD_ERR_ARG, "%s[%lld] is %g, expected 0 or 1", name, (long long)i, a[i]);
    return BBPD_OK;
}

// BONDLIST row q holds two distinct node ids in [1, nN]
inline bool bond_row_ok(const double *bl, int64_t nB, int64_t nN, int64_t q)
{
    const double a = bl[q], b = bl[nB + q];
    return a >= 1 && b >= 1 && a <= (double)nN && b <= (double)nN && a == std::floor(a) && b == std::floor(b) && a != b;
}

static int bad_bond_row(const double *bl, int64_t nB, int64_t k)
{
    return fail(BBPD_ERR_ARG, "BONDLIST row %lld = (%g, %g) is not a pair of distinct node ids", (long long)k + 1, bl[k],
                bl[nB + k]);
}

// Phases of bbpd_create, printed to stderr when BBPD_TIMING is set; each
// phase also waits for the device work it queued unless BBPD_TIMING=nosync.
struct PhaseTimer {
    bool on = std::getenv("BBPD_TIMING") != nullptr;
    bool sync = on && std::strcmp(std::getenv("BBPD_TIMING"), "nosync") != 0;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    void mark(const char *name)
    {
        if (!on) return;
        if (sync) cudaDeviceSynchronize();
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "bbpd_create %-16s %8.1f ms\n", name,
                     std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

// Layout built on the host, for the tiled node order: besides the slices it
// needs each tile's halo list and per-entry local neighbour indices.
template <class FwdIds>
static int host_layout(bbpd_solver *S, const bbpd_problem *pb, const int32_t *inv, FwdIds fwd_ids,
                       const std::vector<uint32_t> &negid, std::vector<DictEntry> &dict, std::vector<float4> &dictx,
                       PhaseTimer &phase)
{
    const bbpd_params *prm = &S->prm;
    const int64_t nN = S->nN, nB = S->nB, ns = S->ns;
    const int T = prm->n_chunks;
    const double *bl = pb->bondlist;
    std::vector<uint32_t> bond_cid(nB), cid_j;
    if (S->prec == kP32X) cid_j.resize(nB);
    const int HT0 = (int)std::min<int64_t>(host_threads(), std::max<int64_t>(1, nB / 65536));
    host_ranges(nB, HT0, [&](int, int64_t lo, int64_t hi) {
        fwd_ids(lo, hi - lo, bond_cid.data() + lo);
        if (S->prec == kP32X)
            for (int64_t k = lo; k < hi; k++) cid_j[k] = negid[bond_cid[k]];
    });
    // per-node lists in bond order, laid out in 32-node slices. Stable
    // counting sort over HT contiguous bond ranges.
    const int HT = (int)std::min<int64_t>(host_threads(), std::max<int64_t>(1, nB / 65536));
    std::vector<std::vector<int32_t>> cnt(HT, std::vector<int32_t>(nN, 0));
    host_ranges(nB, HT, [&](int t, int64_t lo, int64_t hi) {
        int32_t *c = cnt[t].data();
        for (int64_t k = lo; k < hi; k++) {
            c[inv[(int64_t)bl[k] - 1]]++;
            c[inv[(int64_t)bl[nB + k] - 1]]++;
        }
    });
    std::vector<int32_t> deg(nN, 0);
    host_parallel_for(nN, [&](int64_t p) {
        int32_t acc = 0;
        for (int t = 0; t < HT; t++) {
            int32_t c = cnt[t][p];
            cnt[t][p] = acc;   // becomes the thread's first rank in node p's list
            acc += c;
        }
        deg[p] = acc;
    });
    std::vector<int64_t> sptr(ns + 1, 0);
    std::vector<int32_t> slen(ns, 0);
    for (int64_t s = 0; s < ns; s++) {
        int m = 0;
        for (int64_t i = s * 32; i < std::min(nN, s * 32 + 32); i++) m = std::max(m, deg[i]);
        m = (m + 3) & ~3;   // whole groups of 4 entries per lane
        slen[s] = m;
        sptr[s + 1] = sptr[s] + (int64_t)m * 32;
    }
    const int64_t ne = sptr[ns];
    S->ne = ne;
    // Entry streams, left uninitialised here: the scatter below writes every
    // real entry and the chunk pass zeroes the padding, both in parallel.
    std::unique_ptr<uint32_t[]> colw(new uint32_t[std::max<int64_t>(ne, 1)]);
    std::unique_ptr<uint16_t[]> cid16;
    std::unique_ptr<uint32_t[]> cid32;
    if (S->wide) cid32.reset(new uint32_t[std::max<int64_t>(ne, 1)]);
    else cid16.reset(new uint16_t[std::max<int64_t>(ne, 1)]);
    std::unique_ptr<uint8_t[]> st(new uint8_t[std::max<int64_t>(ne, 1)]);
    std::unique_ptr<int32_t[]> bond_of(new int32_t[std::max<int64_t>(ne, 1)]);
    std::vector<double> s0e, s1e, sce;
    if (pb->s0) s0e.assign(ne, 0.0);
    if (pb->s1) s1e.assign(ne, 0.0);
    if (pb->sc || S->wide) sce.assign(ne, prm->sc);   // 32-bit-index instances always read a stream
    S->ent_i.reset(new int64_t[std::max<int64_t>(nB, 1)]);
    S->ent_j.reset(new int64_t[std::max<int64_t>(nB, 1)]);
    host_ranges(nB, HT, [&](int t, int64_t lo, int64_t hi) {
        int32_t *rank = cnt[t].data();
        for (int64_t k = lo; k < hi; k++) {
            const int64_t a = inv[(int64_t)bl[k] - 1], b = inv[(int64_t)bl[nB + k] - 1];
            const uint32_t bt = pb->bond_type ? (uint32_t)pb->bond_type[k] << BT_SHIFT : 0u;
            const uint8_t st0 = (pb->fail && pb->fail[k] == 0) ? ST_BROKEN : 0;
            for (int side = 0; side < 2; side++) {
                const int64_t me = side ? b : a, other = side ? a : b;
                const int64_t pos = entry_pos(sptr[me / 32], rank[me], (int)(me % 32));
                rank[me]++;
                colw[pos] = (uint32_t)other | bt;
                const uint32_t cidv = (side && S->prec == kP32X) ? cid_j[k] : bond_cid[k];
                if (S->wide) cid32[pos] = cidv;
                else cid16[pos] = (uint16_t)cidv;
                st[pos] = st0;
                bond_of[pos] = (int32_t)k;
                if (pb->s0) s0e[pos] = pb->s0[k];
                if (pb->s1) s1e[pos] = pb->s1[k];
                if (pb->sc) sce[pos] = pb->sc[k];
                (side ? S->ent_j : S->ent_i)[k] = pos;
            }
        }
    });
    phase.mark("slices");
    // chunk starts: an entry whose bond lies in another OpenMP chunk than the
    // previous entry of the same list; padding slots (up to the slice's list
    // length, lanes past the last node included) are zeroed
    host_parallel_for(ns * 32, [&](int64_t me) {
        int prev = -1;
        const int32_t dme = me < nN ? deg[me] : 0;
        for (int32_t r = 0; r < dme; r++) {
            const int64_t pos = entry_pos(sptr[me / 32], r, (int)(me % 32));
            const int c = chunk_of_host(bond_of[pos], nB, T);
            if (c != prev) colw[pos] |= F_CHUNK;
            prev = c;
        }
        for (int32_t r = dme; r < slen[me / 32]; r++) {
            const int64_t pos = entry_pos(sptr[me / 32], r, (int)(me % 32));
            colw[pos] = 0;
            if (S->wide) cid32[pos] = 0;
            else cid16[pos] = 0;
            st[pos] = 0;
        }
    });
    bond_of.reset();
    cnt.clear();

    phase.mark("chunk starts");
    // Tiles for the tiled kernel: per tile the sorted list of outside nodes its
    // entries read, and per entry a 12-bit index into [tile nodes, halo].
    std::vector<uint16_t> jw;
    std::vector<int64_t> hptr;
    std::vector<uint32_t> halo;
    int tile_cap = 0;
    if (prm->node_order == BBPD_ORDER_TILED && !S->wide) {
        const int64_t ntiles = (nN + kTile - 1) / kTile;
        std::vector<std::vector<uint32_t>> hl(ntiles);
        std::vector<int> over(HT, 0), capt(HT, 0);
        host_ranges(ntiles, HT, [&](int th, int64_t lo, int64_t hi) {
            for (int64_t t = lo; t < hi; t++) {
                const int64_t n0 = t * kTile, n1 = std::min(nN, n0 + kTile);
                std::vector<uint32_t> &h = hl[t];
                for (int64_t me = n0; me < n1; me++)
                    for (int32_t r = 0; r < deg[me]; r++) {
                        const uint32_t j = colw[entry_pos(sptr[me / 32], r, (int)(me % 32))] & COL_MASK;
                        if ((int64_t)j < n0 || (int64_t)j >= n1) h.push_back(j);
                    }
                std::sort(h.begin(), h.end());
                h.erase(std::unique(h.begin(), h.end()), h.end());
                const int loc = (int)(n1 - n0) + (int)h.size();
                if (loc > kTileCapMax) over[th] = 1;
                capt[th] = std::max(capt[th], loc);
            }
        });
        bool fits = true;
        for (int th = 0; th < HT; th++) {
            fits = fits && !over[th];
            tile_cap = std::max(tile_cap, capt[th]);
        }
        tile_cap = (tile_cap + 31) & ~31;
        int optin = 0;
        BBPD_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, S->device));
        const int ncache = (int)std::min<int64_t>(kDictCache, (int64_t)dict.size());
        const size_t smem = (size_t)32 * ncache + (size_t)24 * tile_cap;
        if (fits && smem <= (size_t)optin) {
            S->tiled = true;
            S->smem = smem;
            jw.assign(ne, 0);
            hptr.assign(ntiles + 1, 0);
            for (int64_t t = 0; t < ntiles; t++) hptr[t + 1] = hptr[t] + (int64_t)hl[t].size();
            halo.resize(hptr[ntiles]);
            host_ranges(ntiles, HT, [&](int, int64_t lo, int64_t hi) {
                for (int64_t t = lo; t < hi; t++) {
                    const int64_t n0 = t * kTile, n1 = std::min(nN, n0 + kTile);
                    const std::vector<uint32_t> &h = hl[t];
                    std::copy(h.begin(), h.end(), halo.begin() + hptr[t]);
                    for (int64_t me = n0; me < n1; me++)
                        for (int32_t r = 0; r < deg[me]; r++) {
                            const int64_t pos = entry_pos(sptr[me / 32], r, (int)(me % 32));
                            const uint32_t w = colw[pos], j = w & COL_MASK;
                            uint32_t l;
                            if ((int64_t)j >= n0 && (int64_t)j < n1) l = (uint32_t)(j - n0);
                            else l = (uint32_t)(n1 - n0) + (uint32_t)(std::lower_bound(h.begin(), h.end(), j) - h.begin());
                            jw[pos] = (uint16_t)(l | ((w & F_CHUNK) ? TF_CHUNK : 0u) |
                                                 (((w >> BT_SHIFT) & 3u) << TBT_SHIFT));
                        }
                }
            });
            // dictionary ordered by use, so that the entries kept in shared
            // memory are the most used ones
            std::vector<int64_t> uses(dict.size(), 0);
            for (int64_t me = 0; me < nN; me++)
                for (int32_t r = 0; r < deg[me]; r++) uses[cid16[entry_pos(sptr[me / 32], r, (int)(me % 32))]]++;
            std::vector<uint32_t> order(dict.size());
            std::iota(order.begin(), order.end(), 0u);
            std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return uses[a] > uses[b]; });
            std::vector<uint32_t> rank(dict.size());
            for (size_t q = 0; q < order.size(); q++) rank[order[q]] = (uint32_t)q;
            for (int64_t e = 0; e < ne; e++) cid16[e] = (uint16_t)rank[cid16[e]];
            std::vector<DictEntry> dict2(dict.size());
            for (size_t q = 0; q < order.size(); q++) dict2[q] = dict[order[q]];
            dict.swap(dict2);
            if (S->prec == kP32X) {
                std::vector<float4> dx2(dictx.size());
                for (size_t q = 0; q < order.size(); q++) {
                    dx2[2 * q] = dictx[2 * order[q]];
                    dx2[2 * q + 1] = dictx[2 * order[q] + 1];
                }
                dictx.swap(dx2);
            }
            S->d.ncache = ncache;
            S->d.tile_cap = tile_cap;
            S->d.n_tiles = ntiles;
        }
    }

    phase.mark("tiles");
    Dev &d = S->d;
    TRY(S->put((int64_t **)&d.slice_ptr, sptr));
    TRY(S->put((int32_t **)&d.deg, deg));
    TRY(S->put((int32_t **)&d.slice_len, slen));
    if (S->tiled) {
        TRY(S->put((uint16_t **)&d.jw, jw));
        TRY(S->put((int64_t **)&d.halo_ptr, hptr));
        TRY(S->put((uint32_t **)&d.halo, halo));
    } else {
        TRY(S->put((uint32_t **)&d.colw, colw.get(), (size_t)ne));
    }
    if (S->wide) TRY(S->put((uint32_t **)&d.cid, cid32.get(), (size_t)ne));
    else TRY(S->put((uint16_t **)&d.cid, cid16.get(), (size_t)ne));
    TRY(S->put(&d.st, st.get(), (size_t)ne));
    TRY(S->alloc(&d.bsf, (size_t)ne));
    BBPD_CUDA_TRY(cudaMemset(d.bsf, 0, sizeof(double) * std::max<int64_t>(ne, 1)));
    if (pb->s0) TRY(S->put((double **)&d.s0e, s0e));
    if (pb->s1) TRY(S->put((double **)&d.s1e, s1e));
    if (pb->sc || S->wide) TRY(S->put((double **)&d.sce, sce));
    return BBPD_OK;
}

// Device buffers that live only while the layout is built, released in
// stream order (no device-wide synchronisation, so other solvers' launches
// keep running while this one is built).
struct TempBufs {
    cudaStream_t st;
    std::vector<void *> p;
    explicit TempBufs(cudaStream_t s) : st(s) {}
    template <class T>
    int get(T **out, size_t count)
    {
        BBPD_CUDA_TRY(cudaMallocAsync((void **)out, sizeof(T) * std::max<size_t>(count, 1), st));
        p.push_back((void *)*out);
        return BBPD_OK;
    }
    ~TempBufs()
    {
        for (void *q : p) cudaFreeAsync(q, st);
    }
};

inline int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

// The layout build's temporaries (gigabytes for large problems) come from the
// device's default stream-ordered pool. With the pool's default release
// threshold of zero, every synchronisation returns the freed memory to the
// driver and the next build maps it again; keeping up to 8 GB reserved lets
// consecutive builds (a serving loop) reuse it. Set once per device.
static void keep_layout_pool(int device)
{
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> g(mu);
    if (std::find(done.begin(), done.end(), device) != done.end()) return;
    done.push_back(device);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = (uint64_t)8 << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
}

// Layout built on the device, for the input and Morton node orders. The host
// converts the per-bond arrays while staging them (node ids to device
// positions, dictionary ids, fail and BONDTYPE packed in a byte); the sort of
// the directed entries by node, the slice shapes and the scatter into the entry
// streams run as kernels, and the bond -> entry map is written on the way.
template <class FwdIds>
static int device_layout(bbpd_solver *S, const bbpd_problem *pb, const int32_t *inv, FwdIds fwd_ids,
                         const std::vector<uint32_t> &negid, PhaseTimer &phase)
{
    const bbpd_params *prm = &S->prm;
    const int64_t nN = S->nN, nB = S->nB, ns = S->ns, n2 = 2 * nB;
    const double *bl = pb->bondlist;
    cudaStream_t st = S->stream;
    Dev &d = S->d;
    keep_layout_pool(S->device);
    TempBufs tmp(st);

    // staged per-bond inputs
    uint32_t *key = nullptr;
    TRY(tmp.get(&key, (size_t)n2));
    // rows are checked on the way (bond_row_ok); the first bad row fails the create
    std::atomic<int64_t> bad_row(nB);
    TRY(staging::upload(key, n2, st, [&](int64_t q0, int64_t cnt, uint32_t *out) {
        int64_t bad = nB;
        for (int64_t i = 0; i < cnt; i++) {
            const int64_t q = q0 + i, k = q >> 1;
            if (!bond_row_ok(bl, nB, nN, k)) {
                bad = std::min(bad, k);
                out[i] = 0;
                continue;
            }
            out[i] = (uint32_t)inv[(int64_t)bl[(q & 1) * nB + k] - 1];
        }
        for (int64_t cur = bad_row.load(); bad < cur && !bad_row.compare_exchange_weak(cur, bad);) {
        }
    }));
    if (bad_row.load() < nB) return bad_bond_row(bl, nB, bad_row.load());
    LayoutArgs a{};
    a.nB = nB;
    a.T = prm->n_chunks;
    a.key = key;
    if (pb->fail || pb->bond_type) {
        uint8_t *bflag = nullptr;
        TRY(tmp.get(&bflag, (size_t)nB));
        const double *fl = pb->fail, *bt = pb->bond_type;
        TRY(staging::upload(bflag, nB, st, [&](int64_t k0, int64_t cnt, uint8_t *out) {
            for (int64_t i = 0; i < cnt; i++) {
                const int64_t k = k0 + i;
                out[i] = (uint8_t)((fl && fl[k] == 0 ? 1 : 0) | (bt ? (int)bt[k] << 1 : 0));
            }
        }));
        a.bflag = bflag;
    }
    if (!S->wide) {
        uint16_t *bcid = nullptr;
        TRY(tmp.get(&bcid, (size_t)nB));
        TRY(staging::upload(bcid, nB, st, [&](int64_t k0, int64_t cnt, uint16_t *out) { fwd_ids(k0, cnt, out); }));
        a.bcid = bcid;
        if (S->prec == kP32X) {
            uint16_t *ng = nullptr;
            TRY(tmp.get(&ng, negid.size()));
            TRY(staging::upload(ng, (int64_t)negid.size(), st, [&](int64_t k0, int64_t cnt, uint16_t *out) {
                for (int64_t i = 0; i < cnt; i++) out[i] = (uint16_t)negid[k0 + i];
            }));
            a.negid = ng;
        }
    }
    const double *lawp[3] = {pb->s0, pb->s1, pb->sc};
    const double **lawd[3] = {&a.s0, &a.s1, &a.sc};
    for (int m = 0; m < 3; m++)
        if (lawp[m]) {
            double *v = nullptr;
            TRY(tmp.get(&v, (size_t)nB));
            TRY(staging::upload_copy(v, lawp[m], nB, st));
            *lawd[m] = v;
        }
    phase.mark("staged bonds");

    // stable sort of the directed entries by node
    uint32_t *skey = nullptr, *val = nullptr, *sval = nullptr;
    TRY(tmp.get(&skey, (size_t)n2));
    TRY(tmp.get(&val, (size_t)n2));
    TRY(tmp.get(&sval, (size_t)n2));
    int end_bit = 1;
    while (end_bit < 32 && ((int64_t)1 << end_bit) < nN) end_bit++;
    if (n2 > 0) {
        k_iota<<<grid_for(n2), 256, 0, st>>>(val, n2);
        BBPD_CUDA_TRY(cudaGetLastError());
        size_t tb = 0;
        BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, skey, val, sval, n2, 0, end_bit, st));
        void *tstore = nullptr;
        TRY(tmp.get((uint8_t **)&tstore, tb));
        BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tstore, tb, key, skey, val, sval, n2, 0, end_bit, st));
    }

    // degrees, slice shapes and offsets
    uint32_t *first = nullptr, *last = nullptr;
    int64_t *scount = nullptr;
    TRY(tmp.get(&first, (size_t)nN));
    TRY(tmp.get(&last, (size_t)nN));
    TRY(tmp.get(&scount, (size_t)ns + 1));
    BBPD_CUDA_TRY(cudaMemsetAsync(first, 0, sizeof(uint32_t) * nN, st));
    BBPD_CUDA_TRY(cudaMemsetAsync(last, 0, sizeof(uint32_t) * nN, st));
    if (n2 > 0) {
        k_run_bounds<<<grid_for(n2), 256, 0, st>>>(skey, n2, first, last);
        BBPD_CUDA_TRY(cudaGetLastError());
    }
    TRY(S->alloc((int32_t **)&d.deg, (size_t)nN));
    TRY(S->alloc((int32_t **)&d.slice_len, (size_t)ns));
    TRY(S->alloc((int64_t **)&d.slice_ptr, (size_t)ns + 1));
    k_slice_lengths<<<grid_for(ns * 32), 256, 0, st>>>(first, last, nN, ns, (int32_t *)d.deg, (int32_t *)d.slice_len,
                                                         scount);
    BBPD_CUDA_TRY(cudaGetLastError());
    {
        size_t tb = 0;
        BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, scount, (int64_t *)d.slice_ptr, ns + 1, st));
        void *tstore = nullptr;
        TRY(tmp.get((uint8_t **)&tstore, tb));
        BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tstore, tb, scount, (int64_t *)d.slice_ptr, ns + 1, st));
    }
    int64_t ne = 0;
    BBPD_CUDA_TRY(cudaMemcpyAsync(&ne, d.slice_ptr + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    S->ne = ne;
    phase.mark("sort, slices");

    // entry streams: padding slots stay zero (the critical stretch stream
    // holds the law's sc there)
    TRY(S->alloc((uint32_t **)&d.colw, (size_t)ne));
    if (S->wide) TRY(S->alloc((uint32_t **)&d.cid, (size_t)ne));
    else TRY(S->alloc((uint16_t **)&d.cid, (size_t)ne));
    TRY(S->alloc(&d.st, (size_t)ne));
    TRY(S->alloc(&d.bsf, (size_t)ne));
    const size_t ne1 = (size_t)std::max<int64_t>(ne, 1);
    BBPD_CUDA_TRY(cudaMemsetAsync((void *)d.colw, 0, 4 * ne1, st));
    BBPD_CUDA_TRY(cudaMemsetAsync((void *)d.cid, 0, (S->wide ? 4 : 2) * ne1, st));
    BBPD_CUDA_TRY(cudaMemsetAsync(d.st, 0, ne1, st));
    BBPD_CUDA_TRY(cudaMemsetAsync(d.bsf, 0, 8 * ne1, st));
    if (pb->s0) {
        TRY(S->alloc((double **)&d.s0e, (size_t)ne));
        BBPD_CUDA_TRY(cudaMemsetAsync((void *)d.s0e, 0, 8 * ne1, st));
    }
    if (pb->s1) {
        TRY(S->alloc((double **)&d.s1e, (size_t)ne));
        BBPD_CUDA_TRY(cudaMemsetAsync((void *)d.s1e, 0, 8 * ne1, st));
    }
    if (pb->sc || S->wide) {   // 32-bit-index instances always read a stream
        TRY(S->alloc((double **)&d.sce, (size_t)ne));
        k_fill<<<grid_for(ne), 256, 0, st>>>((double *)d.sce, ne, prm->sc);
        BBPD_CUDA_TRY(cudaGetLastError());
    }
    S->ent32 = ne < ((int64_t)1 << 32);
    if (S->ent32) TRY(S->alloc((uint32_t **)&S->d_ent, (size_t)n2));
    else TRY(S->alloc((int64_t **)&S->d_ent, (size_t)n2));
    phase.mark("entry streams");
    if (n2 > 0) {
        a.skey = skey;
        a.sval = sval;
        a.first = first;
        a.sptr = d.slice_ptr;
        a.colw = (uint32_t *)d.colw;
        a.cid = (void *)d.cid;
        a.st = d.st;
        a.s0e = (double *)d.s0e;
        a.s1e = (double *)d.s1e;
        a.sce = (double *)d.sce;
        a.ent = S->d_ent;
        a.ent32 = S->ent32 ? 1 : 0;
        k_layout_scatter<<<grid_for(n2), 256, 0, st>>>(a);
        BBPD_CUDA_TRY(cudaGetLastError());
    }
    phase.mark("scatter");
    return BBPD_OK;
}

// ---- lattice form: bond slots (see lstep_kernel) ----

// Bond k into its slot: state byte (fail, BONDTYPE), dictionary id, per-bond
// critical stretch; slot_bond records which bond a slot holds.
__global__ void k_lattice_scatter(int64_t nB, const uint32_t *__restrict__ slot, const uint8_t *__restrict__ bflag,
                                  const uint16_t *__restrict__ bcid, const double *__restrict__ bsc, uint8_t *st,
                                  uint16_t *cid, double *sce, uint32_t *slot_bond)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nB; k += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t q = slot[k];
        if (slot_bond) slot_bond[q] = (uint32_t)k;
        if (st) st[q] = bflag ? bflag[k] : (uint8_t)0;
        if (cid) cid[q] = bcid[k];
        if (sce) sce[q] = bsc[k];
    }
}

// Chain positions of node n whose entry opens a new OpenMP chunk of the
// nodal-force loop (the chunk of its bond differs from that of the node's
// previous entry), packed 8 bits each; *overflow when a node has more than 8.
__global__ void k_lattice_chunks(int64_t nN, int nsig, const int4 *__restrict__ tab,
                                 const uint32_t *__restrict__ slot_bond, int64_t nB, int T, uint64_t *cpos,
                                 int *overflow)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nN; n += (int64_t)gridDim.x * blockDim.x) {
        uint64_t packed = ~0ull;
        int cnt = 0, prev = -1;
        for (int sig = 0; sig < nsig; sig++) {
            const int4 t = tab[sig];
            const int64_t lo = n + t.z;
            if ((uint64_t)lo >= (uint64_t)nN) continue;
            const uint32_t k = slot_bond[(int64_t)t.y + lo];
            if (k == 0xFFFFFFFFu) continue;
            const int c = omp_chunk_of((int64_t)k, nB, T);
            if (prev >= 0 && c != prev) {
                if (cnt == 8) {
                    atomicOr(overflow, 1);
                } else {
                    packed = (packed & ~(0xFFull << (8 * cnt))) | ((uint64_t)sig << (8 * cnt));
                    cnt++;
                }
            }
            prev = c;
        }
        cpos[n] = packed;
    }
}

// Lattice form (BBPD_ORDER_LATTICE). Builds the bond slots when the input is a
// regular lattice in x-fastest order (coordinates bit-equal along every lattice
// row, column and plane) whose bond list is ordered by its first node, with
// the second node after the first and every node's family in one common order
// of stencil offsets; S->lattice stays false otherwise, and nothing is built.
template <class FwdIds>
static int lattice_layout(bbpd_solver *S, const bbpd_problem *pb, FwdIds fwd_ids, std::vector<DictEntry> &dict,
                          PhaseTimer &phase)
{
    S->lattice = false;
    const bbpd_params *prm = &S->prm;
    const int64_t nN = S->nN, nB = S->nB;
    if (S->prec != kP64 || S->wide || pb->s0 || pb->s1 || nB == 0 || dict.size() > 65535) return BBPD_OK;
    const double *X = pb->undeformed_coordinates, *Y = X + nN, *Z = X + 2 * nN;
    int64_t nx = 1;
    while (nx < nN && X[nx] > X[nx - 1]) nx++;
    int64_t ny = 1;
    while (ny * nx < nN && Y[ny * nx] > Y[(ny - 1) * nx]) ny++;
    if (nN % (nx * ny)) return BBPD_OK;
    const int64_t nz = nN / (nx * ny), pl = nx * ny;
    if (nx > 32767 || ny > 32767 || nz > 32767) return BBPD_OK;
    for (int64_t c = 1; c < nz; c++)
        if (!(Z[c * pl] > Z[(c - 1) * pl])) return BBPD_OK;
    const int HT = (int)std::min<int64_t>(host_threads(), std::max<int64_t>(1, nB / 65536));
    {
        std::atomic<bool> ok(true);
        host_ranges(nN, HT, [&](int, int64_t lo, int64_t hi) {
            for (int64_t n = lo; n < hi && ok.load(std::memory_order_relaxed); n++) {
                const int64_t a = n % nx, b = (n / nx) % ny, c = n / pl;
                if (bits_of(X[n]) != bits_of(X[a]) || bits_of(Y[n]) != bits_of(Y[b * nx]) ||
                    bits_of(Z[n]) != bits_of(Z[c * pl]))
                    ok = false;
            }
        });
        if (!ok) return BBPD_OK;
    }
    // pass 1 over the bonds: rows, order, stencil offsets (|component| <= 4)
    const double *bl = pb->bondlist;
    constexpr int KR = 4, KW = 2 * KR + 1, NKEY = KW * KW * KW;
    auto grid_off = [&](int64_t i, int64_t j, int &ox, int &oy, int &oz) {
        ox = (int)(j % nx - i % nx);
        oy = (int)((j / nx) % ny - (i / nx) % ny);
        oz = (int)(j / pl - i / pl);
    };
    std::vector<std::vector<char>> seen(HT, std::vector<char>(NKEY, 0));
    std::atomic<int64_t> bad_row(nB);
    std::atomic<bool> lat(true);
    host_ranges(nB, HT, [&](int t, int64_t lo, int64_t hi) {
        for (int64_t k = lo; k < hi; k++) {
            if (!bond_row_ok(bl, nB, nN, k)) {
                int64_t cur = bad_row.load();
                while (k < cur && !bad_row.compare_exchange_weak(cur, k)) {
                }
                return;
            }
            const int64_t i = (int64_t)bl[k] - 1, j = (int64_t)bl[nB + k] - 1;
            if (j <= i || (k > 0 && bl[k] < bl[k - 1])) { lat = false; return; }
            int ox, oy, oz;
            grid_off(i, j, ox, oy, oz);
            if (std::abs(ox) > KR || std::abs(oy) > KR || std::abs(oz) > KR) { lat = false; return; }
            seen[t][(ox + KR) + KW * ((oy + KR) + KW * (oz + KR))] = 1;
        }
    });
    if (bad_row.load() < nB) return bad_bond_row(bl, nB, bad_row.load());
    if (!lat) return BBPD_OK;
    std::vector<int> fidx_of(NKEY, -1);
    std::vector<int3> foff;
    for (int key = 0; key < NKEY; key++) {
        bool any = false;
        for (int t = 0; t < HT; t++) any |= seen[t][key] != 0;
        if (!any) continue;
        fidx_of[key] = (int)foff.size();
        foff.push_back(make_int3(key % KW - KR, (key / KW) % KW - KR, key / (KW * KW) - KR));
    }
    const int NF = (int)foff.size();
    if (NF > 64 || (int64_t)NF * nN >= ((int64_t)1 << 31)) return BBPD_OK;
    // pass 2: forward offset index per bond, order of offsets within families
    // (an edge a -> b when b follows a in some family), dictionary id use
    std::unique_ptr<uint8_t[]> bf(new uint8_t[nB]);
    std::vector<std::vector<uint64_t>> edge(HT, std::vector<uint64_t>(NF, 0));
    std::vector<std::vector<uint32_t>> use(HT, std::vector<uint32_t>(dict.size(), 0));
    std::unique_ptr<uint16_t[]> bcid(new uint16_t[nB]);
    host_ranges(nB, HT, [&](int t, int64_t lo, int64_t hi) {
        fwd_ids(lo, hi - lo, bcid.get() + lo);
        for (int64_t k = lo; k < hi; k++) {
            const int64_t i = (int64_t)bl[k] - 1, j = (int64_t)bl[nB + k] - 1;
            int ox, oy, oz;
            grid_off(i, j, ox, oy, oz);
            bf[k] = (uint8_t)fidx_of[(ox + KR) + KW * ((oy + KR) + KW * (oz + KR))];
            use[t][bcid[k]]++;
        }
        for (int64_t k = std::max<int64_t>(lo, 1); k < hi; k++) {
            if (bl[k] != bl[k - 1]) continue;
            const int64_t i = (int64_t)bl[k] - 1;
            int ox, oy, oz;
            grid_off(i, (int64_t)bl[nB + k - 1] - 1, ox, oy, oz);
            const int a = fidx_of[(ox + KR) + KW * ((oy + KR) + KW * (oz + KR))];
            grid_off(i, (int64_t)bl[nB + k] - 1, ox, oy, oz);
            const int b = fidx_of[(ox + KR) + KW * ((oy + KR) + KW * (oz + KR))];
            edge[t][a] |= 1ull << b;
        }
    });
    // family order: a topological order of the offsets (smallest index first
    // among the free ones); a cycle, or an offset twice in one family (a
    // self-edge), means no common order
    std::vector<uint64_t> E(NF, 0);
    for (int t = 0; t < HT; t++)
        for (int a = 0; a < NF; a++) E[a] |= edge[t][a];
    std::vector<int> indeg(NF, 0), pi;
    for (int a = 0; a < NF; a++) {
        if (E[a] >> a & 1) return BBPD_OK;
        for (int b = 0; b < NF; b++)
            if (E[a] >> b & 1) indeg[b]++;
    }
    std::vector<char> done(NF, 0);
    for (int r = 0; r < NF; r++) {
        int pick = -1;
        for (int a = 0; a < NF && pick < 0; a++)
            if (!done[a] && indeg[a] == 0) pick = a;
        if (pick < 0) return BBPD_OK;
        done[pick] = 1;
        pi.push_back(pick);
        for (int b = 0; b < NF; b++)
            if (E[pick] >> b & 1) indeg[b]--;
    }
    // chain order: the bonds to lower nodes by ascending partner (the list is
    // ordered by first node), then the node's own family in family order
    int H = 0;
    for (const int3 &f : foff) H = std::max({H, std::abs(f.x), std::abs(f.y), std::abs(f.z)});
    // tile shape: 32 x ty x tz with ty * tz = 8 rows, least padding
    int bty = 4, btz = 2;
    {
        int64_t best = -1;
        const int cand[4][2] = {{4, 2}, {8, 1}, {2, 4}, {1, 8}};
        for (auto &c : cand) {
            const int64_t pad = ((ny + c[0] - 1) / c[0]) * c[0] * ((nz + c[1] - 1) / c[1]) * c[1];
            if (best < 0 || pad < best) { best = pad; bty = c[0]; btz = c[1]; }
        }
    }
    const int lsx = 32 + 2 * H, lsy = bty + 2 * H, lsz = btz + 2 * H;
    auto lin = [&](const int3 &f) { return (int64_t)f.x + nx * ((int64_t)f.y + ny * (int64_t)f.z); };
    // slot rows: one per forward offset plus an all-absent row for the table's
    // padding entries, each padded by the stencil's reach M on both sides
    int64_t M = 0;
    for (const int3 &f : foff) M = std::max<int64_t>(M, lin(f));
    const int64_t R = nN + 2 * M;
    if ((int64_t)(NF + 1) * R >= ((int64_t)1 << 31)) return BBPD_OK;
    std::vector<int> back(NF);
    std::iota(back.begin(), back.end(), 0);
    std::sort(back.begin(), back.end(), [&](int a, int b) { return lin(foff[a]) > lin(foff[b]); });
    std::vector<int4> tab;
    for (int a : back) {
        const int3 &f = foff[a];
        tab.push_back(make_int4(-(f.x + lsx * (f.y + lsy * f.z)), (int)(a * R + M), (int)-lin(f), 0));
    }
    for (int a : pi) {
        const int3 &f = foff[a];
        tab.push_back(make_int4(f.x + lsx * (f.y + lsy * f.z), (int)(a * R + M), 0, 0));
    }
    while (tab.size() % 4) tab.push_back(make_int4(0, (int)(NF * R + M), 0, 0));   // padding: the absent row
    const int nsig = (int)tab.size();
    if (nsig > kMaxSigma) return BBPD_OK;
    // shared memory: positions of the staged box and as many of the most used
    // dictionary entries as fit two blocks per SM
    const size_t box = (size_t)lsx * lsy * lsz;
    const size_t fixed = 24 * box;
    const size_t budget = 110 * 1024;
    if (fixed > budget) return BBPD_OK;
    const int ncache = (int)std::min<size_t>({(size_t)kDictCache, dict.size(), (budget - fixed) / 32});
    // dictionary renumbered by use, most used first (those are cached)
    std::vector<uint32_t> cnt(dict.size(), 0);
    for (int t = 0; t < HT; t++)
        for (size_t c = 0; c < dict.size(); c++) cnt[c] += use[t][c];
    std::vector<uint32_t> order(dict.size());
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cnt[a] > cnt[b]; });
    std::vector<uint16_t> remap(dict.size());
    for (size_t q = 0; q < order.size(); q++) remap[order[q]] = (uint16_t)q;
    phase.mark("lattice check");

    // staged per-bond data, chunk positions, then the slots
    cudaStream_t st = S->stream;
    Dev &d = S->d;
    keep_layout_pool(S->device);
    TempBufs tmp(st);
    const int64_t NS = (int64_t)(NF + 1) * R;
    uint32_t *slot = nullptr, *slot_bond = nullptr;
    TRY(tmp.get(&slot, (size_t)nB));
    TRY(staging::upload(slot, nB, st, [&](int64_t k0, int64_t c, uint32_t *out) {
        for (int64_t q = 0; q < c; q++) {
            const int64_t k = k0 + q;
            out[q] = (uint32_t)((int64_t)bf[k] * R + M + (int64_t)bl[k] - 1);
        }
    }));
    TRY(tmp.get(&slot_bond, (size_t)NS));
    BBPD_CUDA_TRY(cudaMemsetAsync(slot_bond, 0xFF, sizeof(uint32_t) * NS, st));
    k_lattice_scatter<<<grid_for(nB), 256, 0, st>>>(nB, slot, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                    slot_bond);
    BBPD_CUDA_TRY(cudaGetLastError());
    int4 *dtab = nullptr;
    TRY(tmp.get(&dtab, tab.size()));
    BBPD_CUDA_TRY(cudaMemcpyAsync(dtab, tab.data(), sizeof(int4) * tab.size(), cudaMemcpyHostToDevice, st));
    uint64_t *cpos = nullptr;
    TRY(tmp.get(&cpos, (size_t)nN));
    int *over = nullptr;
    TRY(tmp.get(&over, 1));
    BBPD_CUDA_TRY(cudaMemsetAsync(over, 0, sizeof(int), st));
    k_lattice_chunks<<<grid_for(nN), 256, 0, st>>>(nN, nsig, dtab, slot_bond, nB, prm->n_chunks, cpos, over);
    BBPD_CUDA_TRY(cudaGetLastError());
    int hover = 0;
    BBPD_CUDA_TRY(cudaMemcpyAsync(&hover, over, sizeof(int), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    if (hover) return BBPD_OK;   // more than 8 chunk starts in some list (many OpenMP chunks)

    uint8_t *bflag = nullptr;
    if (pb->fail || pb->bond_type) {
        TRY(tmp.get(&bflag, (size_t)nB));
        const double *fl = pb->fail, *btp = pb->bond_type;
        TRY(staging::upload(bflag, nB, st, [&](int64_t k0, int64_t c, uint8_t *out) {
            for (int64_t q = 0; q < c; q++) {
                const int64_t k = k0 + q;
                out[q] = (uint8_t)((fl && fl[k] == 0 ? ST_BROKEN : 0) | (btp ? (int)btp[k] << LST_BT_SHIFT : 0));
            }
        }));
    }
    uint16_t *dcid = nullptr;
    TRY(tmp.get(&dcid, (size_t)nB));
    TRY(staging::upload(dcid, nB, st, [&](int64_t k0, int64_t c, uint16_t *out) {
        for (int64_t q = 0; q < c; q++) out[q] = remap[bcid[k0 + q]];
    }));
    double *dsc = nullptr;
    if (pb->sc) {
        TRY(tmp.get(&dsc, (size_t)nB));
        TRY(staging::upload_copy(dsc, pb->sc, nB, st));
    }
    // from here on the lattice form is committed: its arrays belong to the
    // solver, and the dictionary takes the new numbering (until here the
    // input-order layout may still be built with the old one)
    {
        std::vector<DictEntry> nd(dict.size());
        for (size_t q = 0; q < order.size(); q++) nd[q] = dict[order[q]];
        dict.swap(nd);
    }
    std::memset(&S->ltab, 0, sizeof(LTab));
    std::copy(tab.begin(), tab.end(), S->ltab.e);
    uint64_t *lcpos = nullptr;
    TRY(S->alloc(&lcpos, (size_t)nN));
    BBPD_CUDA_TRY(cudaMemcpyAsync(lcpos, cpos, sizeof(uint64_t) * nN, cudaMemcpyDeviceToDevice, st));
    d.lcpos = lcpos;
    TRY(S->alloc(&d.st, (size_t)NS));
    BBPD_CUDA_TRY(cudaMemsetAsync(d.st, LST_ABSENT, (size_t)NS, st));
    uint16_t *lcid = nullptr;
    TRY(S->alloc(&lcid, (size_t)NS));
    BBPD_CUDA_TRY(cudaMemsetAsync(lcid, 0, 2 * (size_t)NS, st));
    d.cid = lcid;
    TRY(S->alloc(&d.bsf, (size_t)NS));
    BBPD_CUDA_TRY(cudaMemsetAsync(d.bsf, 0, 8 * (size_t)NS, st));
    if (pb->sc) {
        TRY(S->alloc((double **)&d.sce, (size_t)NS));
        k_fill<<<grid_for(NS), 256, 0, st>>>((double *)d.sce, NS, prm->sc);
        BBPD_CUDA_TRY(cudaGetLastError());
    }
    k_lattice_scatter<<<grid_for(nB), 256, 0, st>>>(nB, slot, bflag, dcid, dsc, d.st, lcid, (double *)d.sce,
                                                    nullptr);
    BBPD_CUDA_TRY(cudaGetLastError());
    // bond -> slot map for per-bond gets and sets (both "copies" are the slot)
    S->ent32 = true;
    TRY(S->alloc((uint32_t **)&S->d_ent, (size_t)(2 * nB)));
    BBPD_CUDA_TRY(cudaMemcpyAsync(S->d_ent, slot, sizeof(uint32_t) * nB, cudaMemcpyDeviceToDevice, st));
    BBPD_CUDA_TRY(cudaMemcpyAsync((uint32_t *)S->d_ent + nB, slot, sizeof(uint32_t) * nB, cudaMemcpyDeviceToDevice, st));
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));

    S->ne = NS;
    S->lattice = true;
    d.n_sigma = nsig;
    d.lnx = (int)nx; d.lny = (int)ny; d.lnz = (int)nz;
    d.lty = bty; d.ltz = btz; d.lhalo = H;
    d.lsx = lsx; d.lsy = lsy; d.lsz = lsz;
    d.ltiles[0] = (nx + 31) / 32;
    d.ltiles[1] = (ny + bty - 1) / bty;
    d.ltiles[2] = (nz + btz - 1) / btz;
    d.ncache = ncache;
    S->smem = 32 * (size_t)ncache + fixed;
    phase.mark("lattice slots");
    return BBPD_OK;
}

extern "C" int bbpd_create(const bbpd_problem *pb, const bbpd_params *prm, int device,
                           bbpd_solver **out)
{
    clear_error();
    if (!pb || !prm || !out) return fail(BBPD_ERR_ARG, "null argument");
    *out = nullptr;
    TRY(require_device());
    PhaseTimer phase;
    const int64_t nN = pb->n_nodes, nB = pb->n_bonds;
    if (nN < 1 || nB < 0) return fail(BBPD_ERR_ARG, "n_nodes must be >= 1 and n_bonds >= 0");
    if (nN >= MAX_NODES) return fail(BBPD_ERR_UNSUPPORTED, "at most %lld nodes per solver", (long long)MAX_NODES - 1);
    if (nB >= ((int64_t)1 << 31)) return fail(BBPD_ERR_UNSUPPORTED, "at most 2^31 - 1 bonds per solver");
    if (!pb->undeformed_coordinates || (nB && (!pb->bondlist || !pb->undeformed_length ||
        !pb->bond_stiffness || !pb->volume_correction)))
        return fail(BBPD_ERR_ARG, "missing coordinates or bond arrays");
    if (prm->law < 0 || prm->law > 3 || prm->scheme < 0 || prm->scheme > 1 || prm->precision < 0 ||
        prm->precision > 1 || prm->n_chunks < 1 || prm->n_chunks > 4096)
        return fail(BBPD_ERR_ARG, "bad law/scheme/precision/n_chunks");
    if (!(prm->failure_functionality == 0.0 || prm->failure_functionality == 1.0))
        return fail(BBPD_ERR_UNSUPPORTED, "failure_functionality must be 0 or 1");
    if (prm->scheme == BBPD_SCHEME_ADR && !pb->mass) return fail(BBPD_ERR_ARG, "ADR needs mass");
    if (prm->scheme == BBPD_SCHEME_EULERCROMER && !pb->density) return fail(BBPD_ERR_ARG, "Euler-Cromer needs density");
    if (prm->amplitude == BBPD_AMP_SMOOTHSTEP && prm->n_time_steps < 2)
        return fail(BBPD_ERR_ARG, "smooth step needs n_time_steps >= 2");
    TRY(validate_01(pb->fail, nB, "fail"));
    TRY(validate_01(pb->constraint_flag, 3 * nN, "CONSTRAINTFLAG"));
    TRY(validate_01(pb->prescribed_flag, 3 * nN, "prescribed flag"));
    if (pb->bond_type) {
        const double *bt = pb->bond_type;
        const int64_t k = first_bad(nB, [&](int64_t q) { return !(bt[q] == 0 || bt[q] == 1 || bt[q] == 2); });
        if (k >= 0) return fail(BBPD_ERR_ARG, "BONDTYPE[%lld] = %g", (long long)k, bt[k]);
    }
    if (pb->stretch_plastic) {
        const double *sp = pb->stretch_plastic;
        if (first_bad(nB, [&](int64_t q) { return sp[q] != 0; }) >= 0)
            return fail(BBPD_ERR_UNSUPPORTED, "non-zero stretchPlastic (steel plasticity) is not on this path");
    }
    const double *bl = pb->bondlist;
    // The FP64 form with a device-built layout checks BONDLIST while staging it
    // (the only earlier pass over it); every other configuration reads it
    // before then and checks it here.
    const bool late_bl_check = prm->node_order != BBPD_ORDER_TILED && prm->precision != BBPD_PREC_FP32;
    if (!late_bl_check) {
        const int64_t k = first_bad(nB, [&](int64_t q) { return !bond_row_ok(bl, nB, nN, q); });
        if (k >= 0) return bad_bond_row(bl, nB, k);
    }

    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return fail(BBPD_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    }
    auto *S = new bbpd_solver;
    std::unique_ptr<bbpd_solver> guard_(S);
    S->device = device;
    S->prm = *prm;
    S->nN = nN;
    S->nB = nB;
    S->has_density = pb->density != nullptr;

    phase.mark("validate");
    // node order
    S->perm.resize(nN);
    S->inv.resize(nN);
    std::iota(S->perm.begin(), S->perm.end(), 0);
    if (prm->node_order == BBPD_ORDER_MORTON || prm->node_order == BBPD_ORDER_TILED) {
        const double *X = pb->undeformed_coordinates;
        double lo[3], hi[3];
        for (int c = 0; c < 3; c++) {
            lo[c] = *std::min_element(X + c * nN, X + (c + 1) * nN);
            hi[c] = *std::max_element(X + c * nN, X + (c + 1) * nN);
        }
        // Quantize on the shortest bond length when that resolves the domain
        // in 21 bits per axis: a regular lattice then maps to its integer
        // indices and aligned Morton blocks are exact bricks (a 512-node tile
        // is an 8 x 8 x 8 brick). Otherwise scale each axis to 21 bits.
        double h = 0;
        for (int64_t k = 0; k < nB; k++) {
            const double l = pb->undeformed_length[k];
            if (l > 0 && std::isfinite(l) && (h == 0 || l < h)) h = l;
        }
        bool lattice = h > 0;
        for (int c = 0; c < 3 && lattice; c++) lattice = (hi[c] - lo[c]) / h < 2097000.0;
        std::vector<uint64_t> key(nN);
        for (int64_t i = 0; i < nN; i++) {
            uint32_t q[3];
            for (int c = 0; c < 3; c++) {
                const double span = hi[c] - lo[c];
                if (lattice) q[c] = (uint32_t)std::floor((X[i + c * nN] - lo[c]) / h + 0.5);
                else q[c] = span > 0 ? (uint32_t)((X[i + c * nN] - lo[c]) / span * 2097151.0) : 0;
            }
            key[i] = morton3(q[0], q[1], q[2]);
        }
        std::stable_sort(S->perm.begin(), S->perm.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
    }
    for (int64_t p = 0; p < nN; p++) S->inv[S->perm[p]] = (int32_t)p;
    const int32_t *inv = S->inv.data();

    phase.mark("node order");
    // Dictionary of the distinct bond constants. The FP32 form keys every
    // directed entry by (L0, VCF, BONDSTIFFNESS, bond vector in FP32) and is
    // kept when those keys fit 16-bit ids; otherwise the key is (L0, VCF,
    // BONDSTIFFNESS), and irregular inputs whose keys do not fit 16 bits get one
    // entry per bond (32-bit ids). Ids follow the sorted order of the keys'
    // bits. One pass over the bonds: each host thread numbers the keys of its
    // bond range in a local map and records every bond's local id; the local
    // ids are remapped to dictionary ids while the bonds are laid out.
    const double *X = pb->undeformed_coordinates;
    auto keyx = [&](int64_t k) {   // forward copy: bond vector X[second] - X[first]
        const int64_t a = (int64_t)bl[k] - 1, b = (int64_t)bl[nB + k] - 1;
        const float fx = (float)(X[b] - X[a]), fy = (float)(X[b + nN] - X[a + nN]),
                    fz = (float)(X[b + 2 * nN] - X[a + 2 * nN]);
        return KeyX{bits_of(pb->undeformed_length[k]), bits_of(pb->volume_correction[k]),
                    bits_of(pb->bond_stiffness[k]), fbits(fx), fbits(fy), fbits(fz)};
    };
    auto key3 = [&](int64_t k) {
        return Key3{bits_of(pb->undeformed_length[k]), bits_of(pb->volume_correction[k]),
                    bits_of(pb->bond_stiffness[k])};
    };
    constexpr size_t kLocalMax = 65536;   // local ids are 16-bit; more keys overflow the dictionary anyway
    const int HT = (int)std::min<int64_t>(host_threads(), std::max<int64_t>(1, nB / 65536));
    std::vector<int64_t> rhi(HT);         // bond range of host thread t: [rhi[t-1], rhi[t])
    for (int t = 0; t < HT; t++) rhi[t] = nB * (t + 1) / HT;
    std::unique_ptr<uint16_t[]> lid(new uint16_t[std::max<int64_t>(nB, 1)]);
    std::vector<std::vector<uint32_t>> remap(HT);   // local id -> dictionary id, per thread
    std::vector<uint32_t> negid;
    std::vector<DictEntry> dict;
    std::vector<float4> dictx;
    // one pass: local maps and local ids; false when some thread overflowed
    auto collect = [&](auto key, auto &local) {
        std::vector<char> over(HT, 0);
        host_ranges(nB, HT, [&](int t, int64_t lo, int64_t hi) {
            auto &m = local[t];
            for (int64_t k = lo; k < hi; k++) {
                const uint32_t v = m.insert(key(k), (uint32_t)m.count);
                if (m.count > kLocalMax) {
                    over[t] = 1;
                    return;
                }
                lid[k] = (uint16_t)v;
            }
        });
        for (char o : over)
            if (o) return false;
        return true;
    };
    S->prec = kP64;
    if (prm->precision == BBPD_PREC_FP32) {
        // The reverse copy's key is the forward key with the bond vector
        // negated (IEEE subtraction is sign-symmetric; a +0 component stays
        // +0), so only forward keys are collected and the reverse ids come from
        // the negation of each dictionary key.
        auto negx = [](uint32_t f) { return (f & 0x7FFFFFFFu) ? (f ^ 0x80000000u) : f; };
        auto neg = [&](const KeyX &q) { return KeyX{q.a, q.b, q.c, negx(q.x), negx(q.y), negx(q.z)}; };
        std::vector<FlatMap<KeyX, KeyXHash>> local(HT);
        bool ok = collect(keyx, local);
        FlatMap<KeyX, KeyXHash> idx;
        for (int t = 0; t < HT && ok; t++) {
            local[t].for_each([&](const KeyX &q, uint32_t) {
                idx.insert(q, 0u);
                idx.insert(neg(q), 0u);
            });
            ok = idx.count <= 65535;
        }
        if (ok) {
            std::vector<KeyX> keys;
            keys.reserve(idx.count);
            idx.for_each([&](const KeyX &q, uint32_t) { keys.push_back(q); });
            std::sort(keys.begin(), keys.end());
            for (size_t q = 0; q < keys.size(); q++) idx.set(keys[q], (uint32_t)q);
            for (int t = 0; t < HT; t++) {
                remap[t].resize(local[t].count);
                local[t].for_each([&](const KeyX &q, uint32_t v) { remap[t][v] = idx.find(q); });
            }
            negid.resize(keys.size());
            for (size_t q = 0; q < keys.size(); q++) negid[q] = idx.find(neg(keys[q]));
            dict.resize(keys.size());
            dictx.resize(2 * keys.size());
            for (size_t q = 0; q < keys.size(); q++) {
                double l0, vcf, bs;
                std::memcpy(&l0, &keys[q].a, 8);
                std::memcpy(&vcf, &keys[q].b, 8);
                std::memcpy(&bs, &keys[q].c, 8);
                dict[q] = make_entry(l0, vcf, bs);
                float xf, yf, zf;
                std::memcpy(&xf, &keys[q].x, 4);
                std::memcpy(&yf, &keys[q].y, 4);
                std::memcpy(&zf, &keys[q].z, 4);
                const double c0 = ((double)xf * xf + (double)yf * yf + (double)zf * zf) - l0 * l0;
                dictx[2 * q] = make_float4(xf, yf, zf, (float)l0);
                dictx[2 * q + 1] = make_float4((float)(bs * prm->cell_volume * vcf), (float)c0,
                                               dict[q].rl0 > 0 ? 1.f : 0.f, 0.f);
            }
            S->prec = kP32X;
        }
    }
    phase.mark("fp32 dictionary");
    if (S->prec != kP32X) {
        std::vector<FlatMap<Key3, Key3Hash>> local(HT);
        bool ok = collect(key3, local);
        FlatMap<Key3, Key3Hash> id3;
        for (int t = 0; t < HT && ok; t++) {
            local[t].for_each([&](const Key3 &q, uint32_t) { id3.insert(q, 0u); });
            ok = id3.count <= 65535;
        }
        if (ok) {
            std::vector<Key3> keys;
            keys.reserve(id3.count);
            id3.for_each([&](const Key3 &q, uint32_t) { keys.push_back(q); });
            std::sort(keys.begin(), keys.end());
            for (size_t q = 0; q < keys.size(); q++) id3.set(keys[q], (uint32_t)q);
            for (int t = 0; t < HT; t++) {
                remap[t].resize(local[t].count);
                local[t].for_each([&](const Key3 &q, uint32_t v) { remap[t][v] = id3.find(q); });
            }
            dict.resize(keys.size());
            for (size_t q = 0; q < keys.size(); q++) {
                double l0, vcf, bs;
                std::memcpy(&l0, &keys[q].a, 8);
                std::memcpy(&vcf, &keys[q].b, 8);
                std::memcpy(&bs, &keys[q].c, 8);
                dict[q] = make_entry(l0, vcf, bs);
            }
        } else {
            // irregular input: one dictionary entry per bond, 32-bit ids
            S->wide = true;
            lid.reset();
            dict.resize(nB);
            host_parallel_for(nB, [&](int64_t k) {
                dict[k] = make_entry(pb->undeformed_length[k], pb->volume_correction[k], pb->bond_stiffness[k]);
            });
        }
        if (dict.empty()) dict.push_back(make_entry(1.0, 0.0, 0.0));
    }
    S->ndict = (int64_t)dict.size();
    // Dictionary ids of the copies of bond k in the list of its first node
    // (the copy in its second node's list has negid[] of it in the FP32 form,
    // the same id otherwise), for bonds k0 .. k0 + cnt - 1.
    auto fwd_ids = [&](int64_t k0, int64_t cnt, auto *out) {
        if (S->wide) {
            for (int64_t i = 0; i < cnt; i++) out[i] = (uint32_t)(k0 + i);
            return;
        }
        int t = (int)(std::upper_bound(rhi.begin(), rhi.end(), k0) - rhi.begin());
        for (int64_t i = 0; i < cnt; i++) {
            const int64_t k = k0 + i;
            while (k >= rhi[t]) t++;
            out[i] = remap[t][lid[k]];
        }
    };

    phase.mark("dictionary");
    const int64_t ns = (nN + 31) / 32;
    S->ns = ns;
    Dev &d = S->d;
    d.n_nodes = nN;
    d.n_slices = ns;
    d.colw = nullptr;
    d.jw = nullptr;
    d.halo_ptr = nullptr;
    d.halo = nullptr;
    d.s0e = d.s1e = d.sce = nullptr;
    d.smax = nullptr;
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    if (prm->node_order == BBPD_ORDER_LATTICE) TRY(lattice_layout(S, pb, fwd_ids, dict, phase));
    if (S->lattice) {
    } else if (prm->node_order == BBPD_ORDER_TILED) {
        TRY(host_layout(S, pb, inv, fwd_ids, negid, dict, dictx, phase));
    } else {
        TRY(device_layout(S, pb, inv, fwd_ids, negid, phase));
    }
    lid.reset();

    // node arrays in device order, staged; the initial displacement and
    // positions are formed on the device (k_node_init)
    const int32_t *perm = S->perm.data();
    bool identity = true;
    for (int64_t p = 0; p < nN && identity; p++) identity = perm[p] == p;
    auto stage_nodes = [&](double *dst, const double *src, int ncomp) -> int {
        if (!src) {
            BBPD_CUDA_TRY(cudaMemsetAsync(dst, 0, sizeof(double) * ncomp * nN, S->stream));
            return BBPD_OK;
        }
        if (identity) return staging::upload_copy(dst, src, ncomp * nN, S->stream);
        return staging::upload(dst, ncomp * nN, S->stream, [&](int64_t e0, int64_t cnt, double *out) {
            int64_t c = e0 / nN, p = e0 - c * nN;
            for (int64_t i = 0; i < cnt; i++) {
                out[i] = src[perm[p] + c * nN];
                if (++p == nN) p = 0, c++;
            }
        });
    };
    TRY(S->alloc((double **)&d.X, (size_t)(3 * nN)));
    TRY(stage_nodes((double *)d.X, pb->undeformed_coordinates, 3));
    TRY(S->alloc((double **)&d.mass, (size_t)nN));
    TRY(stage_nodes((double *)d.mass, pb->mass, 1));
    TRY(S->alloc((double **)&d.rho, (size_t)nN));
    TRY(stage_nodes((double *)d.rho, pb->density, 1));
    {
        std::vector<uint8_t> nflag(nN);
        host_parallel_for(nN, [&](int64_t p) {
            const int64_t i = perm[p];
            uint8_t f = 0;
            for (int c = 0; c < 3; c++) {
                const bool cf = pb->constraint_flag && pb->constraint_flag[i + c * nN] == 1;
                const bool pf = pb->prescribed_flag && pb->prescribed_flag[i + c * nN] == 1;
                if (cf || pf) f |= (uint8_t)(1 << c);
                if (pf) f |= (uint8_t)(8 << c);
            }
            nflag[p] = f;
        });
        TRY(S->put((uint8_t **)&d.nflag, nflag));
    }
    phase.mark("node staging");
    double U1;
    if (prm->amplitude == BBPD_AMP_SMOOTHSTEP) {
        // prescribed value at step 1, same arithmetic as the device
        double xi = (1.0 - 1.0) / ((double)prm->n_time_steps - 1.0);
        U1 = 0.0 + (prm->applied_final - 0.0) * ((xi * xi) * xi) * (10 - 15 * xi + 6 * (xi * xi));
    } else {
        U1 = prm->rate * 1.0;
    }
    const size_t b3 = sizeof(double) * 3 * (size_t)nN;
    TRY(S->alloc(&d.xb0, (size_t)(3 * nN)));
    TRY(S->alloc(&d.xb1, (size_t)(3 * nN)));
    TRY(S->alloc(&d.xa0, (size_t)nN));
    TRY(S->alloc(&d.xa1, (size_t)nN));
    TRY(S->alloc(&d.u, (size_t)(3 * nN)));
    TRY(S->alloc(&d.v, (size_t)(3 * nN)));
    TRY(S->alloc(&d.F0, (size_t)(3 * nN)));
    TRY(S->alloc(&d.F1, (size_t)(3 * nN)));
    BBPD_CUDA_TRY(cudaMemsetAsync(d.v, 0, b3, S->stream));
    BBPD_CUDA_TRY(cudaMemsetAsync(d.F0, 0, b3, S->stream));
    BBPD_CUDA_TRY(cudaMemsetAsync(d.F1, 0, b3, S->stream));
    d.a = nullptr;
    if (prm->scheme == BBPD_SCHEME_EULERCROMER) {
        TRY(S->alloc(&d.a, (size_t)(3 * nN)));
        BBPD_CUDA_TRY(cudaMemsetAsync(d.a, 0, b3, S->stream));
    }
    d.urh0 = d.urh1 = nullptr;
    d.url0 = d.url1 = nullptr;
    if (S->prec == kP32X) {
        TRY(S->alloc(&d.urh0, (size_t)nN));
        TRY(S->alloc(&d.urh1, (size_t)nN));
        TRY(S->alloc(&d.url0, (size_t)nN));
        TRY(S->alloc(&d.url1, (size_t)nN));
    }
    TRY(S->alloc(&d.sticky, 1));
    BBPD_CUDA_TRY(cudaMemsetAsync(d.sticky, 0, sizeof(unsigned), S->stream));
    k_node_init<<<grid_for(nN), 256, 0, S->stream>>>(d, U1);
    BBPD_CUDA_TRY(cudaGetLastError());
    phase.mark("node arrays");

    TRY(S->put((DictEntry **)&d.dict, dict));
    d.dictx = nullptr;
    if (S->prec == kP32X) TRY(S->put((float4 **)&d.dictx, dictx));
    {
        // levels of the reduction tree: level 1 has one value per slice,
        // level L+1 one per group of 32 values of level L
        int64_t off = 0, coff = 0, c = ns;
        int L = 1;
        d.lvl_cnt[L] = c;
        d.lvl_off[L] = 0;
        d.cnt_off[L] = 0;
        off = c;
        while (c > 1) {
            if (L + 1 >= kMaxLevels) return fail(BBPD_ERR_UNSUPPORTED, "too many slices for the reduction tree");
            c = (c + 31) / 32;
            L++;
            d.lvl_cnt[L] = c;
            d.lvl_off[L] = off;
            d.cnt_off[L] = coff;
            off += c;
            coff += c;
        }
        d.n_levels = L;
        TRY(S->alloc(&d.tree, (size_t)std::max<int64_t>(off, 1)));
        TRY(S->alloc(&d.tree3, (size_t)std::max<int64_t>(off, 1)));
        std::vector<unsigned> tc((size_t)std::max<int64_t>(coff, 1), 0u);
        TRY(S->put(&d.tcnt, tc));
    }
    d.react_cap = kReactCap;
    TRY(S->alloc(&d.react, (size_t)kReactCap));
    BBPD_CUDA_TRY(cudaMemset(d.react, 0, sizeof(double) * kReactCap));
    d.law = prm->law;
    d.prec = S->prec;
    std::vector<double> sc4(4, 0.0);
    TRY(S->put(&d.scal, sc4));
    std::vector<unsigned> bar(2, 0u);
    TRY(S->put(&d.bar, bar));
    std::vector<unsigned long long> work(1, 0ull);
    TRY(S->put(&d.work, work));
    std::vector<int> err(1, 0);
    TRY(S->put(&d.err, err));

    phase.mark("uploads");
    // scalars
    LawScalars &P = d.P;
    P.s0 = prm->s0; P.s1 = prm->s1; P.sc = prm->sc;
    // FP32 fast-path s0: an entry whose stretch exceeds the least per-bond s0
    // goes to the general path, which reads its own s0 (NaN values are
    // skipped; an all-NaN array gives NaN, which like each NaN s0 keeps every
    // entry quiet)
    d.s0q = prm->s0;
    if (pb->s0 && nB > 0) {
        double m = NAN;
        for (int64_t k = 0; k < nB; k++) m = std::fmin(m, pb->s0[k]);
        d.s0q = m;
    }
    P.beta = prm->beta_tri;
    double eta = prm->s1 / prm->s0;
    P.tri_c1 = (eta - P.beta) / (eta - 1);
    P.tri_c2 = (1 - P.beta) / (eta - 1);
    P.k = prm->k_exp;
    P.alpha = prm->alpha_exp;
    P.exp_den = 1 - std::exp(-prm->k_exp);
    P.sc_steel = prm->sc_steel;
    P.ff = prm->failure_functionality;
    d.V = prm->cell_volume;
    d.dt = prm->dt;
    d.damping = prm->damping;
    d.amplitude = prm->amplitude;
    d.rate = prm->rate;
    d.applied_final = prm->applied_final;
    d.n_time_steps = prm->n_time_steps;
    d.guard = prm->guard_band;
    double to = prm->barrier_timeout_s > 0 ? prm->barrier_timeout_s : 2.0;
    d.timeout_ns = (unsigned long long)(to * 1e9);

    // kernel and grid
    if (S->lattice) {
        S->kernel = reinterpret_cast<kernel_t>(pick_lkernel(prm->law, prm->scheme, pb->sc != nullptr));
        BBPD_CUDA_TRY(cudaFuncSetAttribute((const void *)S->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)S->smem));
    } else if (S->tiled) {
        S->kernel = pick_tkernel(prm->law, prm->scheme, S->prec, pb->sc != nullptr);
        BBPD_CUDA_TRY(cudaFuncSetAttribute((const void *)S->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)S->smem));
    } else {
        S->kernel = pick_kernel(prm->law, prm->scheme, S->prec, S->wide, pb->sc != nullptr);
    }
    int nsm = 0, occ = 0, coop = 0;
    BBPD_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    BBPD_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    if (!coop) return fail(BBPD_ERR_UNSUPPORTED, "device lacks cooperative launch");
    BBPD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void *)S->kernel, kBlock, S->smem));
    if (occ < 1) return fail(BBPD_ERR_CUDA, "kernel cannot be resident");
    int64_t want = (ns * 32 + kBlock - 1) / kBlock;   // one warp per slice at most
    S->grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)nsm * occ, want));
    BBPD_CUDA_TRY(cudaEventCreate(&S->ev0));
    BBPD_CUDA_TRY(cudaEventCreate(&S->ev1));

    // DRAM bytes one step moves with this layout (streams of the live entries,
    // node arrays; dictionary and damaged-bond BSF reads excluded)
    {
        double per_entry = (S->tiled ? 2 : 4) + (S->wide ? 4 : 2) + 1 + (pb->s0 ? 8 : 0) + (pb->s1 ? 8 : 0) + (pb->sc ? 8 : 0);
        // lattice form: each bond slot (state byte, dictionary id, sc) read once from DRAM
        if (S->lattice) per_entry = 0.5 * (double)S->ne / (double)std::max<int64_t>(nB, 1) * (2 + 1 + (pb->sc ? 8 : 0));
        double node = prm->scheme == BBPD_SCHEME_ADR
                          ? (24 /*x*/ + 4 /*deg*/ + 24 * 3 + 8 /*u v Fp m*/ + 24 /*F w*/ +
                             24 * 4 + 8 + 1 /*F u v X m flag*/ + 72 /*v u x w*/)
                          : (24 + 4 + 24 * 3 + 8 + 1 /*x v u X rho flag*/ + 24 * 5 /*F a v u x w*/);
        S->bytes_per_step = 2.0 * (double)nB * per_entry + (double)nN * node;
    }
    // the layout and staged copies ran on this solver's stream, the small
    // uploads on the legacy default stream; wait for those only, not for
    // other solvers' launches on their own streams
    phase.mark("kernel setup");
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    BBPD_CUDA_TRY(cudaStreamSynchronize(0));
    *out = guard_.release();
    return BBPD_OK;
}

static int collect_status(bbpd_solver *S)
{
    int h = 0;
    BBPD_CUDA_TRY(cudaMemcpyAsync(&h, S->d.err, sizeof(int), cudaMemcpyDeviceToHost, S->stream));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (h) {
        int z = 0;
        BBPD_CUDA_TRY(cudaMemcpy(S->d.err, &z, sizeof(int), cudaMemcpyHostToDevice));
        if (h & ERR_TIMEOUT) return fail(BBPD_ERR_TIMEOUT, "grid barrier wait exceeded its limit; kernel returned early");
        return fail(BBPD_ERR_NONFINITE, "non-finite displacement or velocity");
    }
    return BBPD_OK;
}

extern "C" int bbpd_step_async(bbpd_solver *S, int64_t nsteps)
{
    if (!S || nsteps < 0) return fail(BBPD_ERR_ARG, "bad argument");
    if (S->batch) return fail(BBPD_ERR_ARG, "solver is a batch member: step it with bbpd_batch_step");
    if (nsteps == 0) return BBPD_OK;
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    int64_t step0 = S->step;
    void *args[] = {(void *)&S->d, (void *)&step0, (void *)&nsteps, (void *)&S->ltab};   // lattice kernels take the table
    BBPD_CUDA_TRY(cudaMemsetAsync(S->d.work, 0, sizeof(unsigned long long), S->stream));
    BBPD_CUDA_TRY(cudaEventRecord(S->ev0, S->stream));
    BBPD_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)S->kernel, dim3(S->grid), dim3(kBlock), args, S->smem, S->stream));
    BBPD_CUDA_TRY(cudaEventRecord(S->ev1, S->stream));
    S->step += nsteps;
    return BBPD_OK;
}

extern "C" int bbpd_sync(bbpd_solver *S)
{
    if (!S) return fail(BBPD_ERR_ARG, "null solver");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    int rc = collect_status(S);
    if (rc) return rc;
    if (S->prm.scheme == BBPD_SCHEME_ADR) {
        BBPD_CUDA_TRY(cudaMemcpy(&S->cn, S->d.scal, sizeof(double), cudaMemcpyDeviceToHost));
    }
    return BBPD_OK;
}

extern "C" int bbpd_step(bbpd_solver *S, int64_t nsteps)
{
    TRY(bbpd_step_async(S, nsteps));
    return bbpd_sync(S);
}

extern "C" int bbpd_last_kernel_ms(bbpd_solver *S, float *ms)
{
    if (!S || !ms) return fail(BBPD_ERR_ARG, "null argument");
    BBPD_CUDA_TRY(cudaEventElapsedTime(ms, S->ev0, S->ev1));
    return BBPD_OK;
}

extern "C" int bbpd_batch_remove(bbpd_batch *B, bbpd_solver *S);

extern "C" int bbpd_destroy(bbpd_solver *S)
{
    if (!S) return BBPD_OK;
    if (S->batch) bbpd_batch_remove(S->batch, S);
    cudaSetDevice(S->device);
    if (S->stream) cudaStreamSynchronize(S->stream);
    delete S;
    return BBPD_OK;
}

static double *field_ptr(bbpd_solver *S, int field, bool &nodal)
{
    Dev &d = S->d;
    nodal = true;
    const int64_t last = S->step - 1;  // last completed step
    switch (field) {
    case BBPD_FIELD_DISPLACEMENT: return d.u;
    case BBPD_FIELD_VELOCITY: return d.v;
    case BBPD_FIELD_FORCE: return (last & 1) ? d.F1 : d.F0;
    case BBPD_FIELD_FORCE_PREV: return (last & 1) ? d.F0 : d.F1;
    case BBPD_FIELD_DEFORMED: return (last & 1) ? d.xb1 : d.xb0;
    case BBPD_FIELD_ACCELERATION: return d.a;
    default: nodal = false; return nullptr;
    }
}

// The bond -> entry map on the device (first per-bond get or set): 32-bit
// positions when the layout allows; the host copy is released after.
static int upload_entry_map(bbpd_solver *S)
{
    if (S->d_ent) return BBPD_OK;
    const int64_t nB = S->nB;
    S->ent32 = S->ne < ((int64_t)1 << 32);
    if (S->ent32) {
        std::vector<uint32_t> m(2 * nB);
        host_parallel_for(nB, [&](int64_t k) {
            m[k] = (uint32_t)S->ent_i[k];
            m[nB + k] = (uint32_t)S->ent_j[k];
        });
        uint32_t *d = nullptr;
        TRY(S->put(&d, m));
        S->d_ent = d;
    } else {
        std::vector<int64_t> m(2 * nB);
        std::copy(S->ent_i.get(), S->ent_i.get() + nB, m.begin());
        std::copy(S->ent_j.get(), S->ent_j.get() + nB, m.begin() + nB);
        int64_t *d = nullptr;
        TRY(S->put(&d, m));
        S->d_ent = d;
    }
    S->ent_i.reset();
    S->ent_j.reset();
    return BBPD_OK;
}

extern "C" int bbpd_get(bbpd_solver *S, int field, double *out)
{
    if (!S || !out) return fail(BBPD_ERR_ARG, "null argument");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    const int64_t nN = S->nN, nB = S->nB;
    bool nodal;
    double *src = field_ptr(S, field, nodal);
    if (nodal) {
        if (!src) return fail(BBPD_ERR_ARG, "field %d not held by this scheme", field);
        const int32_t *perm = S->perm.data();
        return staging::download(src, 3 * nN, S->stream, [&](int64_t e0, int64_t cnt, const double *in) {
            int64_t c = e0 / nN, p = e0 - c * nN;
            for (int64_t i = 0; i < cnt; i++) {
                out[perm[p] + c * nN] = in[i];
                if (++p == nN) p = 0, c++;
            }
        });
    }
    if (field == BBPD_FIELD_DAMAGE_ENERGY) {
        if (!S->d.smax) return fail(BBPD_ERR_ARG, "damage energy is not tracked (bbpd_track_damage_energy)");
        if (nB == 0) return BBPD_OK;
        TRY(upload_entry_map(S));
        // calculatedamageenergy.m:36 and its shape factor, formed once with the host's exp
        const double k = S->prm.k_exp, alpha = S->prm.alpha_exp, V = S->prm.cell_volume;
        const double ek = std::exp(k);
        const double den = 2 * k * (ek - 1) * (1 + alpha);
        const double shape = (2 * k) - (2 * ek) + (alpha * k) - (alpha * k * ek) + 2;
        const Dev &d = S->d;
        const int blocks = (int)std::min<int64_t>((nB + 255) / 256, 148 * 32);
        double *tmp = nullptr;
        BBPD_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(double) * (size_t)nB, S->stream));
        const void *ent = S->d_ent;
        if (S->ent32 && !S->wide)
            k_bond_energy<uint32_t, uint16_t><<<blocks, 256, 0, S->stream>>>((const uint32_t *)ent, nB, d.smax,
                (const uint16_t *)d.cid, d.dict, d.s0e, d.sce, d.P.s0, d.P.sc, shape, den, V * V, tmp);
        else if (S->ent32)
            k_bond_energy<uint32_t, uint32_t><<<blocks, 256, 0, S->stream>>>((const uint32_t *)ent, nB, d.smax,
                (const uint32_t *)d.cid, d.dict, d.s0e, d.sce, d.P.s0, d.P.sc, shape, den, V * V, tmp);
        else if (!S->wide)
            k_bond_energy<int64_t, uint16_t><<<blocks, 256, 0, S->stream>>>((const int64_t *)ent, nB, d.smax,
                (const uint16_t *)d.cid, d.dict, d.s0e, d.sce, d.P.s0, d.P.sc, shape, den, V * V, tmp);
        else
            k_bond_energy<int64_t, uint32_t><<<blocks, 256, 0, S->stream>>>((const int64_t *)ent, nB, d.smax,
                (const uint32_t *)d.cid, d.dict, d.s0e, d.sce, d.P.s0, d.P.sc, shape, den, V * V, tmp);
        cudaError_t e = cudaGetLastError();
        int rc = e == cudaSuccess ? BBPD_OK : fail(BBPD_ERR_CUDA, "damage energy: %s", cudaGetErrorString(e));
        if (rc == BBPD_OK) rc = staging::download_copy(out, tmp, nB, S->stream);
        cudaFreeAsync(tmp, S->stream);
        return rc;
    }
    if (field != BBPD_FIELD_BSF && field != BBPD_FIELD_FLAG && field != BBPD_FIELD_FAIL)
        return fail(BBPD_ERR_ARG, "unknown field %d", field);
    if (nB == 0) return BBPD_OK;
    TRY(upload_entry_map(S));
    const int blocks = (int)std::min<int64_t>((nB + 255) / 256, 148 * 32);
    if (field != BBPD_FIELD_BSF) {   // 0/1 values cross as bytes
        uint8_t *tb = nullptr;
        BBPD_CUDA_TRY(cudaMallocAsync(&tb, (size_t)nB, S->stream));
        if (S->ent32)
            k_bond_gather_bits<uint32_t><<<blocks, 256, 0, S->stream>>>((const uint32_t *)S->d_ent, nB, S->d.st, field, tb);
        else
            k_bond_gather_bits<int64_t><<<blocks, 256, 0, S->stream>>>((const int64_t *)S->d_ent, nB, S->d.st, field, tb);
        cudaError_t e = cudaGetLastError();
        int rc = e == cudaSuccess ? BBPD_OK : fail(BBPD_ERR_CUDA, "get field %d: %s", field, cudaGetErrorString(e));
        if (rc == BBPD_OK)
            rc = staging::download(tb, nB, S->stream, [&](int64_t k0, int64_t cnt, const uint8_t *in) {
                for (int64_t i = 0; i < cnt; i++) out[k0 + i] = (double)in[i];
            });
        cudaFreeAsync(tb, S->stream);
        return rc;
    }
    double *tmp = nullptr;
    BBPD_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(double) * (size_t)nB, S->stream));
    if (S->ent32)
        k_bond_gather<uint32_t><<<blocks, 256, 0, S->stream>>>((const uint32_t *)S->d_ent, nB, S->d.bsf, S->d.st, field, tmp);
    else
        k_bond_gather<int64_t><<<blocks, 256, 0, S->stream>>>((const int64_t *)S->d_ent, nB, S->d.bsf, S->d.st, field, tmp);
    cudaError_t e = cudaGetLastError();
    int rc = e == cudaSuccess ? BBPD_OK : fail(BBPD_ERR_CUDA, "get field %d: %s", field, cudaGetErrorString(e));
    if (rc == BBPD_OK) rc = staging::download_copy(out, tmp, nB, S->stream);
    cudaFreeAsync(tmp, S->stream);
    return rc;
}

extern "C" int bbpd_set(bbpd_solver *S, int field, const double *in)
{
    if (!S || !in) return fail(BBPD_ERR_ARG, "null argument");
    if (S->batch) TRY(batch_member_changed(S->batch));
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    const int64_t nN = S->nN, nB = S->nB;
    bool nodal;
    double *dst = field_ptr(S, field, nodal);
    if (nodal) {
        if (!dst) return fail(BBPD_ERR_ARG, "field %d not held by this scheme", field);
        std::vector<double> h(3 * nN);
        for (int c = 0; c < 3; c++)
            for (int64_t p = 0; p < nN; p++) h[p + c * nN] = in[S->perm[p] + c * nN];
        BBPD_CUDA_TRY(cudaMemcpy(dst, h.data(), sizeof(double) * 3 * nN, cudaMemcpyHostToDevice));
        if (field == BBPD_FIELD_DISPLACEMENT && S->prec == kP32X) {
            // the FP32 form gathers an FP32 record of the displacement
            std::vector<float4> uh;
            std::vector<float2> ul;
            split_record(h.data(), nN, uh, ul);
            BBPD_CUDA_TRY(cudaMemcpy(S->d.urh0, uh.data(), sizeof(float4) * nN, cudaMemcpyHostToDevice));
            BBPD_CUDA_TRY(cudaMemcpy(S->d.urh1, uh.data(), sizeof(float4) * nN, cudaMemcpyHostToDevice));
            BBPD_CUDA_TRY(cudaMemcpy(S->d.url0, ul.data(), sizeof(float2) * nN, cudaMemcpyHostToDevice));
            BBPD_CUDA_TRY(cudaMemcpy(S->d.url1, ul.data(), sizeof(float2) * nN, cudaMemcpyHostToDevice));
        }
        if (field == BBPD_FIELD_DEFORMED) {
            // both position buffers: the next step reads the one of its parity
            BBPD_CUDA_TRY(cudaMemcpy(dst == S->d.xb0 ? S->d.xb1 : S->d.xb0, h.data(), sizeof(double) * 3 * nN, cudaMemcpyHostToDevice));
            // the position records follow, ordered after those copies on the
            // legacy stream
            const int blocks = (int)std::min<int64_t>((nN + 255) / 256, 148 * 32);
            k_pack_positions<<<blocks, 256, 0, 0>>>(S->d.xb0, nN, S->d.xa0);
            k_pack_positions<<<blocks, 256, 0, 0>>>(S->d.xb1, nN, S->d.xa1);
            BBPD_CUDA_TRY(cudaGetLastError());
            BBPD_CUDA_TRY(cudaStreamSynchronize(0));
            bool far = false;
            for (double x : h) far |= !coord_safe(x);
            if (far) {   // sticky: from now on the kernels divide with IEEE division
                const unsigned one = 1u;
                BBPD_CUDA_TRY(cudaMemcpy(S->d.sticky, &one, sizeof(unsigned), cudaMemcpyHostToDevice));
            }
        }
        return BBPD_OK;
    }
    if (field != BBPD_FIELD_BSF && field != BBPD_FIELD_FLAG && field != BBPD_FIELD_FAIL)
        return fail(BBPD_ERR_ARG, "unknown field %d", field);
    if (field != BBPD_FIELD_BSF) TRY(validate_01(in, nB, field == BBPD_FIELD_FLAG ? "flagBondSoftening" : "fail"));
    if (nB == 0) return BBPD_OK;
    TRY(upload_entry_map(S));
    double *tmp = nullptr;
    BBPD_CUDA_TRY(cudaMallocAsync(&tmp, sizeof(double) * (size_t)nB, S->stream));
    const int rc = staging::upload_copy(tmp, in, nB, S->stream);
    if (rc) {
        cudaFreeAsync(tmp, S->stream);
        return rc;
    }
    cudaError_t e = cudaSuccess;
    const int blocks = (int)std::min<int64_t>((nB + 255) / 256, 148 * 32);
    {
        if (S->ent32)
            k_bond_scatter<uint32_t><<<blocks, 256, 0, S->stream>>>((const uint32_t *)S->d_ent, nB, tmp, field, S->d.bsf, S->d.st);
        else
            k_bond_scatter<int64_t><<<blocks, 256, 0, S->stream>>>((const int64_t *)S->d_ent, nB, tmp, field, S->d.bsf, S->d.st);
        e = cudaGetLastError();
    }
    cudaFreeAsync(tmp, S->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "set field %d: %s", field, cudaGetErrorString(e));
    return BBPD_OK;
}

extern "C" int bbpd_track_damage_energy(bbpd_solver *S)
{
    if (!S) return fail(BBPD_ERR_ARG, "null solver");
    if (S->prm.law == BBPD_LAW_LINEAR)
        return fail(BBPD_ERR_UNSUPPORTED, "damage energy is tracked for the softening laws only");
    if (S->batch) TRY(batch_member_changed(S->batch));
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (!S->d.smax) TRY(S->alloc(&S->d.smax, (size_t)S->ne));
    BBPD_CUDA_TRY(cudaMemsetAsync(S->d.smax, 0, sizeof(double) * (size_t)std::max<int64_t>(S->ne, 1), S->stream));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    return BBPD_OK;
}

extern "C" int bbpd_get_step(bbpd_solver *S, int64_t *step, double *cn)
{
    if (!S) return fail(BBPD_ERR_ARG, "null solver");
    if (S->cn_stale) {   // last stepped by a batch launch
        BBPD_CUDA_TRY(cudaSetDevice(S->device));
        BBPD_CUDA_TRY(cudaMemcpy(&S->cn, S->d.scal, sizeof(double), cudaMemcpyDeviceToHost));
        S->cn_stale = false;
    }
    if (step) *step = S->step;
    if (cn) *cn = S->cn;
    return BBPD_OK;
}

extern "C" int bbpd_set_step(bbpd_solver *S, int64_t step, double cn)
{
    if (!S || step < 1) return fail(BBPD_ERR_ARG, "bad argument");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    // F and position buffers are addressed by step parity: keep their contents
    // attached to the right step when the parity changes
    if (((step - S->step) & 1) != 0) {
        std::swap(S->d.F0, S->d.F1);
        std::swap(S->d.xb0, S->d.xb1);
        std::swap(S->d.xa0, S->d.xa1);
        std::swap(S->d.urh0, S->d.urh1);
        std::swap(S->d.url0, S->d.url1);
    }
    S->step = step;
    S->cn = cn;
    S->cn_stale = false;
    if (S->batch) TRY(batch_member_changed(S->batch));
    BBPD_CUDA_TRY(cudaMemcpy(S->d.scal, &cn, sizeof(double), cudaMemcpyHostToDevice));
    return BBPD_OK;
}

extern "C" int bbpd_selftest_wait_timeout(double timeout_s)
{
    TRY(require_device());
    if (!(timeout_s > 0 && timeout_s <= 5)) return fail(BBPD_ERR_ARG, "timeout must be in (0, 5] s");
    unsigned *word = nullptr;
    int *err = nullptr;
    BBPD_CUDA_TRY(cudaMalloc(&word, sizeof(unsigned)));
    BBPD_CUDA_TRY(cudaMalloc(&err, sizeof(int)));
    BBPD_CUDA_TRY(cudaMemset(word, 0, sizeof(unsigned)));
    BBPD_CUDA_TRY(cudaMemset(err, 0, sizeof(int)));
    wait_selftest_kernel<<<1, 32>>>(word, err, (unsigned long long)(timeout_s * 1e9));
    cudaError_t e = cudaDeviceSynchronize();
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(word);
    cudaFree(err);
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "selftest: %s", cudaGetErrorString(e));
    if (h & ERR_TIMEOUT) return fail(BBPD_ERR_TIMEOUT, "bounded wait expired as expected");
    return BBPD_OK;
}

extern "C" int bbpd_get_info(bbpd_solver *S, bbpd_info *info)
{
    if (!S || !info) return fail(BBPD_ERR_ARG, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->n_nodes = S->nN;
    info->n_bonds = S->nB;
    info->n_entries = S->ne;
    info->n_slices = S->ns;
    info->grid_blocks = S->grid;
    info->block_threads = kBlock;
    info->device_bytes = S->device_bytes;
    info->bytes_per_step = S->bytes_per_step;
    info->layout = (S->wide ? 2 : (S->prec == kP32X ? 3 : 1)) + (S->tiled ? 16 : 0) + (S->lattice ? 32 : 0);
    info->reserved = (int32_t)std::min<int64_t>(S->ndict, INT32_MAX);
    return BBPD_OK;
}

// ------------------------------------------------------------------ batches

// One class of batch members: same law and kernel precision variant, stepped
// by one persistent launch of its own specialised kernel.
struct BatchClass {
    int law = 0, prec = kP64;
    bool sce = false;                        // members read a per-entry critical stretch
    batch_kernel_t kernel = nullptr;
    std::vector<bbpd_solver *> members;
    Dev *d_members = nullptr;
    int64_t *d_prefix = nullptr, *d_mstep = nullptr;
    size_t cap = 0;
    unsigned long long *work = nullptr;
    int occ = 0;
    BatchCtl ctl{};

    void release()
    {
        for (void *p : {(void *)d_members, (void *)d_prefix, (void *)d_mstep, (void *)work})
            if (p) cudaFree(p);
        d_members = nullptr;
        d_prefix = d_mstep = nullptr;
        work = nullptr;
        cap = 0;
    }
};

struct bbpd_batch {
    int device = 0;
    int prec = kP64;                       // kP64: FP64 members; kP32X: FP32 members (either FP32 variant)
    std::vector<bbpd_solver *> members;
    bool dirty = true;                     // class tables must be rebuilt before the next launch
    std::vector<BatchClass> classes;       // non-empty classes of the current membership
    unsigned *bar = nullptr;
    int *err = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int nsm = 0, occ = 0;                  // SMs, resident blocks per SM (smallest over the kernels)
    int blocks_per_sm = 0;                 // schedule: resident blocks used per SM
    int grab = 1;                          // schedule: slices per counter grab
    bool tuned = false;
    int64_t total = 0;
    double timeout_s = 2.0;
    bool use_graph = true;                 // replay the launches from a captured CUDA graph
    bool mixed = false;                    // true: all laws of a precision variant in one launch
    bool mixing_fixed = false;             // set by bbpd_batch_set_mixing; else the tuner chooses
    cudaGraphExec_t gexec = nullptr;
    int64_t g_nsteps = -1;
    int g_bps = 0, g_grab = 0;
    bool last_graph = false;

    void drop_graph()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
        g_nsteps = -1;
    }
    ~bbpd_batch()
    {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        drop_graph();
        for (BatchClass &c : classes) c.release();
        for (void *p : {(void *)bar, (void *)err})
            if (p) cudaFree(p);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
        for (bbpd_solver *S : members) S->batch = nullptr;
    }
};

static int batch_member_changed(bbpd_batch *B)
{
    BBPD_CUDA_TRY(cudaSetDevice(B->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(B->stream));
    B->dirty = true;
    return BBPD_OK;
}

extern "C" int bbpd_batch_create(int device, int precision, bbpd_batch **out)
{
    clear_error();
    if (!out || (precision != BBPD_PREC_FP64 && precision != BBPD_PREC_FP32)) return fail(BBPD_ERR_ARG, "bad argument");
    *out = nullptr;
    TRY(require_device());
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return fail(BBPD_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    }
    auto *B = new bbpd_batch;
    std::unique_ptr<bbpd_batch> guard_(B);
    B->device = device;
    B->prec = precision == BBPD_PREC_FP32 ? kP32X : kP64;
    BBPD_CUDA_TRY(cudaMalloc((void **)&B->bar, 2 * sizeof(unsigned)));
    BBPD_CUDA_TRY(cudaMemset(B->bar, 0, 2 * sizeof(unsigned)));
    BBPD_CUDA_TRY(cudaMalloc((void **)&B->err, sizeof(int)));
    BBPD_CUDA_TRY(cudaMemset(B->err, 0, sizeof(int)));
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    BBPD_CUDA_TRY(cudaEventCreate(&B->ev0));
    BBPD_CUDA_TRY(cudaEventCreate(&B->ev1));
    int coop = 0;
    BBPD_CUDA_TRY(cudaDeviceGetAttribute(&B->nsm, cudaDevAttrMultiProcessorCount, device));
    BBPD_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    if (!coop) return fail(BBPD_ERR_UNSUPPORTED, "device lacks cooperative launch");
    // resident blocks per SM: the smallest over the kernels this batch may run
    int occ = 1 << 30;
    for (int law = 0; law < 4; law++)
        for (int pv : {kP64, kP32X}) {
            if (pv == kP32X && B->prec == kP64) continue;
            for (bool sce : {false, true}) {
                int o = 0;
                BBPD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, (const void *)pick_batch_kernel(law, pv, sce), kBlock, 0));
                occ = std::min(occ, o);
            }
        }
    for (int pv : {kP64, kP32X}) {
        if (pv == kP32X && B->prec == kP64) continue;
        int o = 0;
        BBPD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, (const void *)pick_batch_mixed(pv), kBlock, 0));
        occ = std::min(occ, o);
    }
    if (occ < 1) return fail(BBPD_ERR_CUDA, "batch kernel cannot be resident");
    B->occ = occ;
    B->blocks_per_sm = occ;
    *out = guard_.release();
    return BBPD_OK;
}

extern "C" int bbpd_batch_destroy(bbpd_batch *B)
{
    delete B;
    return BBPD_OK;
}

extern "C" int bbpd_batch_add(bbpd_batch *B, bbpd_solver *S)
{
    if (!B || !S) return fail(BBPD_ERR_ARG, "null argument");
    if (S->batch) return fail(BBPD_ERR_ARG, "solver already belongs to a batch");
    if (S->device != B->device) return fail(BBPD_ERR_ARG, "solver and batch live on different devices");
    if (S->prm.scheme != BBPD_SCHEME_ADR) return fail(BBPD_ERR_UNSUPPORTED, "batches run the ADR scheme");
    if (S->prm.precision != (B->prec == kP64 ? BBPD_PREC_FP64 : BBPD_PREC_FP32))
        return fail(BBPD_ERR_UNSUPPORTED, "solver precision form differs from the batch's");
    if (S->wide || S->tiled || S->lattice)
        return fail(BBPD_ERR_UNSUPPORTED, "batch members need 16-bit dictionary ids and input or Morton node order");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    BBPD_CUDA_TRY(cudaStreamSynchronize(B->stream));
    B->members.push_back(S);
    S->batch = B;
    B->dirty = true;
    return BBPD_OK;
}

extern "C" int bbpd_batch_remove(bbpd_batch *B, bbpd_solver *S)
{
    if (!B || !S) return fail(BBPD_ERR_ARG, "null argument");
    auto it = std::find(B->members.begin(), B->members.end(), S);
    if (it == B->members.end()) return fail(BBPD_ERR_ARG, "solver is not a member of this batch");
    BBPD_CUDA_TRY(cudaSetDevice(B->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(B->stream));
    B->members.erase(it);
    S->batch = nullptr;
    B->dirty = true;
    return BBPD_OK;
}

// Class tables (member descriptors, slice prefix, step numbers) of the
// current membership: one class per precision variant (and per law and
// critical-stretch form when mixing is off), members in the order they joined.
static int batch_rebuild(bbpd_batch *B)
{
    std::vector<BatchClass> old;
    old.swap(B->classes);
    for (bbpd_solver *S : B->members) {
        BatchClass *c = nullptr;
        // one class per kernel precision variant (every law in one launch),
        // or, with mixing off, per law and critical-stretch form as well
        const bool sce = B->mixed ? false : S->d.sce != nullptr;
        const int law = B->mixed ? -1 : S->prm.law;
        for (BatchClass &k : B->classes)
            if (k.law == law && k.prec == S->prec && k.sce == sce) c = &k;
        if (!c) {
            B->classes.emplace_back();
            c = &B->classes.back();
            c->law = law;
            c->prec = S->prec;
            c->sce = sce;
            c->kernel = B->mixed ? pick_batch_mixed(c->prec) : pick_batch_kernel(c->law, c->prec, sce);
            // reuse the device tables of the same class from before
            for (BatchClass &o : old)
                if (o.law == c->law && o.prec == c->prec && o.sce == c->sce && o.cap) {
                    c->d_members = o.d_members;
                    c->d_prefix = o.d_prefix;
                    c->d_mstep = o.d_mstep;
                    c->work = o.work;
                    c->cap = o.cap;
                    o.cap = 0;
                    o.d_members = nullptr;
                    o.d_prefix = o.d_mstep = nullptr;
                    o.work = nullptr;
                }
        }
        c->members.push_back(S);
    }
    for (BatchClass &o : old) o.release();
    B->drop_graph();
    B->total = 0;
    double to = 0;
    for (BatchClass &c : B->classes) {
        const size_t S = c.members.size();
        if (S > c.cap) {
            c.release();
            const size_t cap = std::max<size_t>(S, 8);
            BBPD_CUDA_TRY(cudaMalloc((void **)&c.d_members, sizeof(Dev) * cap));
            BBPD_CUDA_TRY(cudaMalloc((void **)&c.d_prefix, sizeof(int64_t) * (cap + 1)));
            BBPD_CUDA_TRY(cudaMalloc((void **)&c.d_mstep, sizeof(int64_t) * cap));
            BBPD_CUDA_TRY(cudaMalloc((void **)&c.work, sizeof(unsigned long long)));
            c.cap = cap;
        }
        std::vector<Dev> devs(S);
        std::vector<int64_t> prefix(S + 1, 0), mstep(S);
        for (size_t m = 0; m < S; m++) {
            devs[m] = c.members[m]->d;
            prefix[m + 1] = prefix[m] + c.members[m]->ns;
            mstep[m] = c.members[m]->step;
            const double t = c.members[m]->prm.barrier_timeout_s;
            to = std::max(to, t > 0 ? t : 2.0);
        }
        BBPD_CUDA_TRY(cudaMemcpy(c.d_members, devs.data(), sizeof(Dev) * S, cudaMemcpyHostToDevice));
        BBPD_CUDA_TRY(cudaMemcpy(c.d_mstep, mstep.data(), sizeof(int64_t) * S, cudaMemcpyHostToDevice));
        BBPD_CUDA_TRY(cudaMemcpy(c.d_prefix, prefix.data(), sizeof(int64_t) * (S + 1), cudaMemcpyHostToDevice));
        c.ctl.members = c.d_members;
        c.ctl.prefix = c.d_prefix;
        c.ctl.mstep = c.d_mstep;
        c.ctl.S = (int)S;
        c.ctl.total = prefix[S];
        c.ctl.bar = B->bar;
        c.ctl.work = c.work;
        c.ctl.err = B->err;
        B->total += prefix[S];
    }
    B->timeout_s = to > 0 ? to : 2.0;
    for (BatchClass &c : B->classes) c.ctl.timeout_ns = (unsigned long long)(B->timeout_s * 1e9);
    B->dirty = false;
    return BBPD_OK;
}

// Enqueue the launches of every class for nsteps steps with the given
// schedule: counter reset and one persistent launch per class.
static int batch_enqueue(bbpd_batch *B, int64_t nsteps, int blocks_per_sm, int grab)
{
    for (BatchClass &c : B->classes) {
        int64_t want = (c.ctl.total * 32 + kBlock - 1) / kBlock;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)B->nsm * blocks_per_sm, want));
        c.ctl.grab = grab;
        void *args[] = {(void *)&c.ctl, (void *)&nsteps};
        BBPD_CUDA_TRY(cudaMemsetAsync(c.work, 0, sizeof(unsigned long long), B->stream));
        BBPD_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)c.kernel, dim3(grid), dim3(kBlock), args, 0, B->stream));
    }
    return BBPD_OK;
}

// Launch nsteps steps of every member: graph replay when enabled and the
// capture succeeds, direct launches otherwise.
static int batch_launch(bbpd_batch *B, int64_t nsteps, int blocks_per_sm, int grab, bool graph)
{
    B->last_graph = false;
    if (graph && B->use_graph) {
        if (!B->gexec || B->g_nsteps != nsteps || B->g_bps != blocks_per_sm || B->g_grab != grab) {
            B->drop_graph();
            cudaGraph_t g = nullptr;
            bool ok = cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                const int rc = batch_enqueue(B, nsteps, blocks_per_sm, grab);
                ok = cudaStreamEndCapture(B->stream, &g) == cudaSuccess && g && rc == BBPD_OK;
            }
            if (ok) ok = cudaGraphInstantiate(&B->gexec, g, 0) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
            if (!ok) {   // capture of these launches is not available here: launch directly from now on
                cudaGetLastError();
                clear_error();
                B->drop_graph();
                B->use_graph = false;
            } else {
                B->g_nsteps = nsteps;
                B->g_bps = blocks_per_sm;
                B->g_grab = grab;
            }
        }
        if (B->gexec) {
            BBPD_CUDA_TRY(cudaEventRecord(B->ev0, B->stream));
            BBPD_CUDA_TRY(cudaGraphLaunch(B->gexec, B->stream));
            BBPD_CUDA_TRY(cudaEventRecord(B->ev1, B->stream));
            B->last_graph = true;
            return BBPD_OK;
        }
    }
    BBPD_CUDA_TRY(cudaEventRecord(B->ev0, B->stream));
    TRY(batch_enqueue(B, nsteps, blocks_per_sm, grab));
    BBPD_CUDA_TRY(cudaEventRecord(B->ev1, B->stream));
    return BBPD_OK;
}

// Wait for the launches, then account them to every member: step numbers, and
// error flags (the batch's barrier flag and each member's own flag).
static int batch_finish(bbpd_batch *B, int64_t nsteps)
{
    BBPD_CUDA_TRY(cudaStreamSynchronize(B->stream));
    int h = 0;
    BBPD_CUDA_TRY(cudaMemcpy(&h, B->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        int z = 0;
        BBPD_CUDA_TRY(cudaMemcpy(B->err, &z, sizeof(int), cudaMemcpyHostToDevice));
        B->dirty = true;   // step numbers on the device may not have advanced
        return fail(BBPD_ERR_TIMEOUT, "batch grid barrier wait exceeded its limit; kernel returned early");
    }
    int bad = -1;
    for (size_t m = 0; m < B->members.size(); m++) {
        bbpd_solver *S = B->members[m];
        S->step += nsteps;
        S->cn_stale = true;
        int e = 0;
        BBPD_CUDA_TRY(cudaMemcpy(&e, S->d.err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e && bad < 0) bad = (int)m;
        if (e) {
            int z = 0;
            BBPD_CUDA_TRY(cudaMemcpy(S->d.err, &z, sizeof(int), cudaMemcpyHostToDevice));
        }
    }
    if (bad >= 0) return fail(BBPD_ERR_NONFINITE, "non-finite displacement or velocity in batch member %d", bad);
    return BBPD_OK;
}

extern "C" int bbpd_batch_step(bbpd_batch *B, int64_t nsteps)
{
    if (!B || nsteps < 0) return fail(BBPD_ERR_ARG, "bad argument");
    if (nsteps == 0 || B->members.empty()) return BBPD_OK;
    BBPD_CUDA_TRY(cudaSetDevice(B->device));
    if (B->dirty) TRY(batch_rebuild(B));
    TRY(batch_launch(B, nsteps, B->blocks_per_sm, B->grab, true));
    return batch_finish(B, nsteps);
}

extern "C" int bbpd_batch_tune(bbpd_batch *B, int64_t nsteps_per_trial, int *blocks_per_sm, int *grab)
{
    if (!B || nsteps_per_trial < 1) return fail(BBPD_ERR_ARG, "bad argument");
    if (B->members.empty()) return fail(BBPD_ERR_ARG, "empty batch");
    BBPD_CUDA_TRY(cudaSetDevice(B->device));
    if (B->dirty) TRY(batch_rebuild(B));
    // Candidate schedules: resident blocks per SM x slices per grab, and,
    // unless the caller fixed it, one launch for all laws or one per law.
    // Every trial runs real steps of the members, so tuning costs no extra
    // work; trials of the same length compare the same steps' work.
    float best = 0;
    int bb = B->occ, bg = 1;
    bool bmix = B->mixed, first = true;
    std::vector<bool> mixes = {B->mixed};
    if (!B->mixing_fixed) mixes = {true, false};
    for (bool mix : mixes) {
        if (mix != B->mixed) {
            B->mixed = mix;
            TRY(batch_rebuild(B));
        }
        for (int bps = 1; bps <= B->occ; bps++)
            for (int g : {1, 2, 4}) {
                TRY(batch_launch(B, nsteps_per_trial, bps, g, false));
                TRY(batch_finish(B, nsteps_per_trial));
                float ms = 0;
                BBPD_CUDA_TRY(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
                if (first || ms < best) {
                    best = ms;
                    bb = bps;
                    bg = g;
                    bmix = mix;
                    first = false;
                }
            }
    }
    if (bmix != B->mixed) {
        B->mixed = bmix;
        TRY(batch_rebuild(B));
    }
    B->blocks_per_sm = bb;
    B->grab = bg;
    B->tuned = true;
    B->drop_graph();
    if (blocks_per_sm) *blocks_per_sm = bb;
    if (grab) *grab = bg;
    return BBPD_OK;
}

extern "C" int bbpd_batch_set_schedule(bbpd_batch *B, int blocks_per_sm, int grab, int use_graph)
{
    if (!B || blocks_per_sm < 1 || grab < 1 || grab > 64) return fail(BBPD_ERR_ARG, "bad argument");
    B->blocks_per_sm = std::min(blocks_per_sm, B->occ);
    B->grab = grab;
    B->use_graph = use_graph != 0;
    B->drop_graph();
    return BBPD_OK;
}

extern "C" int bbpd_batch_set_mixing(bbpd_batch *B, int mixed)
{
    if (!B) return fail(BBPD_ERR_ARG, "null batch");
    TRY(batch_member_changed(B));
    B->mixed = mixed != 0;
    B->mixing_fixed = true;
    return BBPD_OK;
}

extern "C" int bbpd_batch_get_info(bbpd_batch *B, bbpd_batch_info *info)
{
    if (!B || !info) return fail(BBPD_ERR_ARG, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->n_members = (int32_t)B->members.size();
    info->blocks_per_sm = B->blocks_per_sm;
    info->grab = B->grab;
    info->graph = B->last_graph ? 1 : 0;
    info->total_slices = B->total;
    info->n_classes = (int32_t)B->classes.size();
    int64_t bytes = 0;
    for (bbpd_solver *S : B->members) bytes += S->device_bytes;
    info->device_bytes = bytes;
    return BBPD_OK;
}

extern "C" int bbpd_batch_last_kernel_ms(bbpd_batch *B, float *ms)
{
    if (!B || !ms) return fail(BBPD_ERR_ARG, "null argument");
    BBPD_CUDA_TRY(cudaEventElapsedTime(ms, B->ev0, B->ev1));
    return BBPD_OK;
}

extern "C" int bbpd_set_contact(bbpd_solver *S, int n, const bbpd_penetrator *pen)
{
    if (!S || n < 0 || n > 4 || (n > 0 && !pen)) return fail(BBPD_ERR_ARG, "bad argument (at most 4 cylinders)");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (S->batch) TRY(batch_member_changed(S->batch));
    Dev &d = S->d;
    if (n == 0) {
        d.n_pen = 0;
        return BBPD_OK;
    }
    if (!S->has_density) return fail(BBPD_ERR_UNSUPPORTED, "contact needs DENSITY (calculatecontactforce.m:80)");
    const int64_t nN = S->nN;
    std::vector<int32_t> cidx(nN, -1);
    int64_t off[5] = {0, 0, 0, 0, 0};
    for (int p = 0; p < n; p++) {
        const bbpd_penetrator &q = pen[p];
        if (!(q.radius > 0) || !std::isfinite(q.radius) || !std::isfinite(q.centre_x) ||
            !std::isfinite(q.centre_z) || !std::isfinite(q.increment) || q.n_family < 0 ||
            (q.n_family > 0 && !q.family))
            return fail(BBPD_ERR_ARG, "cylinder %d: bad centre, radius, increment or family", p);
        off[p + 1] = off[p] + q.n_family;
        for (int64_t f = 0; f < q.n_family; f++) {
            const double id = q.family[f];
            if (!(id >= 1 && id <= (double)nN && id == std::floor(id)))
                return fail(BBPD_ERR_ARG, "cylinder %d: family[%lld] = %g is not a node id", p, (long long)f, id);
            const int32_t dev = S->inv[(int64_t)id - 1];
            if (cidx[dev] >= 0)
                return fail(BBPD_ERR_UNSUPPORTED, "node %g is in two cylinder families (families must be disjoint)", id);
            cidx[dev] = (int32_t)(off[p] + f);
        }
    }
    const int64_t ntot = off[n];
    std::vector<double> cz(8, 0.0), zero(2 * std::max<int64_t>(ntot, 1), 0.0);
    for (int p = 0; p < n; p++) cz[p] = cz[4 + p] = pen[p].centre_z;
    int32_t *dcidx = nullptr;
    double *dcf = nullptr, *dcz = nullptr;
    TRY(S->put(&dcidx, cidx));
    TRY(S->put(&dcf, zero));
    TRY(S->put(&dcz, cz));
    d.cidx = dcidx;
    d.cforce = dcf;
    d.pen_cz = dcz;
    d.n_contact = ntot;
    for (int p = 0; p < 4; p++) {
        const bool on = p < n;
        d.pen_cx[p] = on ? pen[p].centre_x : 0.0;
        d.pen_r[p] = on ? pen[p].radius : 0.0;
        d.pen_inc[p] = on ? pen[p].increment : 0.0;
        d.pen_react[p] = on ? (pen[p].reaction != 0) : 0;
    }
    for (int p = 0; p <= 4; p++) d.pen_off[p] = off[std::min(p, n)];
    d.n_pen = n;
    return BBPD_OK;
}

extern "C" int bbpd_set_probes(bbpd_solver *S, int n, const double *node_ids, const int32_t *dofs)
{
    if (!S || n < 0 || n > 8 || (n > 0 && (!node_ids || !dofs))) return fail(BBPD_ERR_ARG, "bad argument (at most 8 probes)");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (S->batch) TRY(batch_member_changed(S->batch));
    Dev &d = S->d;
    for (int k = 0; k < n; k++) {
        const double id = node_ids[k];
        if (!(id >= 1 && id <= (double)S->nN && id == std::floor(id)) || dofs[k] < 0 || dofs[k] > 2)
            return fail(BBPD_ERR_ARG, "probe %d: node %g / dof %d out of range", k, id, dofs[k]);
    }
    if (n > 0 && !d.probe_hist) {
        double *h = nullptr;
        TRY(S->alloc(&h, (size_t)(8 * kReactCap)));
        BBPD_CUDA_TRY(cudaMemset(h, 0, sizeof(double) * 8 * kReactCap));
        d.probe_hist = h;
    }
    for (int k = 0; k < 8; k++) {
        d.probe_node[k] = k < n ? S->inv[(int64_t)node_ids[k] - 1] : -1;
        d.probe_dof[k] = k < n ? dofs[k] : 0;
    }
    d.n_probe = n;
    return BBPD_OK;
}

extern "C" int bbpd_get_probes(bbpd_solver *S, int64_t nsteps, double *out)
{
    if (!S || !out || nsteps < 0) return fail(BBPD_ERR_ARG, "bad argument");
    if (nsteps > kReactCap) return fail(BBPD_ERR_ARG, "at most %lld steps of probes are kept", (long long)kReactCap);
    if (S->d.n_probe == 0) return fail(BBPD_ERR_ARG, "no probes set");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (S->batch) TRY(batch_member_changed(S->batch));
    if (nsteps)
        BBPD_CUDA_TRY(cudaMemcpy(out, S->d.probe_hist, sizeof(double) * (size_t)(nsteps * S->d.n_probe),
                                 cudaMemcpyDeviceToHost));
    return BBPD_OK;
}

extern "C" int bbpd_get_reaction(bbpd_solver *S, int64_t n, double *out)
{
    if (!S || !out || n < 0) return fail(BBPD_ERR_ARG, "bad argument");
    if (S->prm.scheme != BBPD_SCHEME_ADR && S->d.n_pen == 0)
        return fail(BBPD_ERR_UNSUPPORTED, "without contact the reaction is summed by the ADR scheme");
    if (n > kReactCap) return fail(BBPD_ERR_ARG, "at most %lld per-step reactions are kept", (long long)kReactCap);
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (S->batch) TRY(batch_member_changed(S->batch));
    if (n) BBPD_CUDA_TRY(cudaMemcpy(out, S->d.react, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return BBPD_OK;
}
