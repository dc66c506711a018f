// Symmetry functions and their derivatives -- kernel templates, instantiated
// per cutoff type and compute type by kernels_sf_*.cu.  R = double is the
// plain form; R = float is the precision form (neighbor displacements are
// FP64 in memory and rounded to FP32 when staged; outputs are FP32).
//
// Semantics: Element::calculateSymmetryFunctionGroups driving
//   SymGrpExpRad::calculate   (libnnp/SymGrpExpRad.cpp:144-239)   type 2
//   SymGrpExpAngn::calculate  (libnnp/SymGrpExpAngn.cpp:156-403)  type 3
//   SymGrpExpAngw::calculate  (libnnp/SymGrpExpAngw.cpp:156-376)  type 9
// with CutoffFunction::fdf (libnnp/CutoffFunction.cpp:128-213) and
// CoreFunction (libnnp/CoreFunction.h:171-320).
//
// Decomposition (B200): one WARP per central atom i (persistent grid).  The
// atom's neighbors are staged in the warp's shared memory, grouped by
// element (the neighbor list is stored element-grouped), with per-neighbor
// quantities computed once: 1/r, f_c, f_c'/r and, per distinct (eta, rs) of
// the angular members, E(r) = exp(-eta (r - rs)^2).  The angular exponential
// of a triplet is then E(r_ij) E(r_ik) exp(-eta (r_jk - rs)^2): the same
// value as the reference's single exp up to rounding.
//
// Work items are (group, owner neighbor j) pairs, flattened over all groups of
// equal (type, rc), 32 per round.  The owner accumulates, over its partners k
// of the group's other element,
//   * its own dG/dr slot:  -(sum_k p1(j,k)) dr_ij - sum_k p3(j,k) (dr_ik - dr_ij)
//     -- kept in registers and written once (single writer, no atomics);
//   * the value 1/2 sum_k term(j,k) (each unordered pair is seen by both
//     owners; 0.5 scales exactly), folded into per-warp sums keyed by
//     symmetry function.
// The self derivative dG/dr_i is not formed: the reference adds to the atom
// exactly what it subtracts from the neighbor slots
// (SymGrpExpRad.cpp:215-226, SymGrpExpAngn.cpp:366-383), so
// dG/dr_i = -sum over entries of the slots, which the force kernel applies
// as minus the sum of the atom's pair terms (and selfDerivativeKernel forms
// on request).
// For j as first member of the pair p1 is the reference's p1, for j as second
// it is the reference's p2 -- the same expression with roles swapped.
// Narrow-angular partners come from a per-atom validity bitmask
// (r_ik < rc, r_jk < rc), so lanes only iterate valid triplets.  All sums are
// formed in a fixed order: results are deterministic run to run.
//
// Product-form fast path.  When a group's members are (eta runs) x (zeta,
// lambda shapes) with integer zeta and rs = 0 (the usual n2p2 layout), the
// reference's per-member expressions (SymGrpExpAngn.cpp:292-336) factor, with
// pfczl * p2etapl = 2 eta pfc plambda, into
//   term = vexp_eta * A_s * plambda_s * pfc,        A_s = plambda_s^(zeta-1)
//   p1   = fn * vexp_eta * A_s * (zl_s X1 + plambda_s (pr1 - 2 eta pfc))
//   p3   = fn * vexp_eta * A_s * (zl_s X3 + plambda_s (2 eta pfc - pr3))
// with X1 = pfc (1/(r_ij r_ik) - cos/r_ij^2), X3 = pfc/(r_ij r_ik), zl = zeta
// lambda and fn the member's 2^(1-zeta) * scaling factor.  Per pair one exp
// per eta run and one power per shape remain; each member costs 9
// operations.  Other groups take the general path, which keeps the
// reference's expression form.
//
// dG/dr layout per atom i (n neighbors, S = maxSlots):
//   dGdr[nbrOff[i]*S*3 + (slot*3 + c)*n + t]
// consecutive neighbors t are consecutive in memory: owner lanes store, and
// the force kernel loads, coalesced.
#pragma once

#include <cstdlib>

#include "device_common.cuh"
#include "kernels.h"

namespace n2p2b
{
namespace sfk
{

constexpr int kWarps = 4;                 // warps (atoms) per CTA

// Bytes of the block-shared group + member tables (16-byte padded); tables
// above kMaxTableBytes stay in global memory (read through L1) instead
// (SFParams::stageTables, set by the host).
constexpr std::size_t kMaxTableBytes = 32 * 1024;
__host__ __device__ inline std::size_t tableBytes(int ng, int nm)
{
    return ((ng * sizeof(DevGroup) + nm * sizeof(DevMember) + 15) / 16) * 16;
}
__host__ __device__ inline std::size_t stagedTableBytes(SFParams const& P)
{
    return P.stageTables ? tableBytes(P.numGroups, P.numMembers) : 0;
}
constexpr int kThreads = 32 * kWarps;
// Members per register chunk of the general paths; small so that their
// register demand stays below the product-form path's.
constexpr int kGenericChunk = 6;
// Members per register chunk of the compact angular path: a whole group of
// up to 8 members in one pass over the triplets (acos, divisions and radial
// values are per triplet, not per member).
constexpr int kCompactChunk = 8;
constexpr unsigned kFull = 0xffffffffu;


// Math in the compute type.  The FP32 (precision) form uses the hardware
// approximations for exp and for the cosine cutoff's sin / cos: relative
// errors of a few 1e-7 at the arguments met here (|x| below ~30 for exp;
// pi x in [0, pi] for the cutoff), far inside the form's stated accuracy.
__device__ __forceinline__ double mexp(double x) { return exp(x); }
__device__ __forceinline__ float mexp(float x) { return __expf(x); }
__device__ __forceinline__ double mtanh(double x) { return tanh(x); }
__device__ __forceinline__ float mtanh(float x) { return tanhf(x); }
__device__ __forceinline__ double mpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float mpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double mrsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float mrsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ void msincospi(double x, double* s, double* c)
{
    sincospi(x, s, c);
}
__device__ __forceinline__ void msincospi(float x, float* s, float* c)
{
    __sincosf(3.14159265358979f * x, s, c);
}

// CutoffFunction::fdf specialized on the (global) cutoff type; CT = -1
// dispatches at run time.
template <typename R, int CT>
__device__ __forceinline__ void cutoffFdf(SFParams const& P, DevGroup const& g,
                                          R r, R& fc, R& dfc);

template <typename R, int CT>
__device__ __forceinline__ void cutoffFdfT(SFParams const& P, DevGroup const& g,
                                           R r, R& fc, R& dfc)
{
    R const rcinv = R(g.rcinv);
    R const iw = R(g.iw);
    if (r >= R(g.rc))
    {
        fc = R(0);
        dfc = R(0);
        return;
    }
    if (CT == 0)
    {
        fc = R(1);
        dfc = R(0);
    }
    else if (CT == 2 || CT == 3)   // CT_TANHU, CT_TANH
    {
        R const temp = mtanh(R(1) - r * rcinv);
        R const temp2 = temp * temp;
        R const pre = (CT == 3) ? R(P.TANH_PRE) : R(1);
        fc = pre * temp * temp2;
        dfc = R(3) * pre * temp2 * (temp2 - R(1)) * rcinv;
    }
    else
    {
        if (r < R(g.rci))
        {
            fc = R(1);
            dfc = R(0);
            return;
        }
        R const x = (r - R(g.rci)) * iw;
        if (CT == 1)               // CT_COS: d/dr cos uses sin(pi x) >= 0
        {
            R s, c;
            msincospi(x, &s, &c);
            fc = R(0.5) * (c + R(1));
            dfc = R(-0.5) * iw * R(P.PI) * s;
        }
        else
        {
            R fx, dfx;
            if (CT == 4)           // CT_EXP
            {
                R const temp = R(1) / (x * x - R(1));
                R const temp2 = mexp(temp);
                fx = R(P.E) * temp2;
                dfx = R(-2) * R(P.E) * x * temp * temp * temp2;
            }
            else if (CT == 5)      // CT_POLY1
            {
                fx = (R(2) * x - R(3)) * x * x + R(1);
                dfx = x * (R(6) * x - R(6));
            }
            else if (CT == 6)      // CT_POLY2
            {
                R const x2 = x * x;
                fx = ((R(15) - R(6) * x) * x - R(10)) * x * x2 + R(1);
                dfx = x2 * ((R(60) - R(30) * x) * x - R(30));
            }
            else if (CT == 7)      // CT_POLY3
            {
                R const x2 = x * x;
                fx = (x * (x * (R(20) * x - R(70)) + R(84)) - R(35)) * x2 * x2
                     + R(1);
                dfx = x2 * x * (x * (x * (R(140) * x - R(420)) + R(420))
                                - R(140));
            }
            else                   // CT_POLY4
            {
                R x4 = x * x;
                x4 *= x4;
                fx = (x * (x * ((R(315) - R(70) * x) * x - R(540)) + R(420))
                      - R(126)) * x * x4 + R(1);
                dfx = x4 * (x * (x * ((R(2520) - R(630) * x) * x - R(3780))
                                 + R(2520)) - R(630));
            }
            fc = fx;
            dfc = dfx * iw;
        }
    }
}

template <typename R, int CT>
__device__ __forceinline__ void cutoffFdf(SFParams const& P, DevGroup const& g,
                                          R r, R& fc, R& dfc)
{
    if (CT >= 0)
    {
        cutoffFdfT<R, (CT >= 0 ? CT : 0)>(P, g, r, fc, dfc);
        return;
    }
    switch (P.cutoffType)
    {
    case 0: cutoffFdfT<R, 0>(P, g, r, fc, dfc); break;
    case 1: cutoffFdfT<R, 1>(P, g, r, fc, dfc); break;
    case 2: cutoffFdfT<R, 2>(P, g, r, fc, dfc); break;
    case 3: cutoffFdfT<R, 3>(P, g, r, fc, dfc); break;
    case 4: cutoffFdfT<R, 4>(P, g, r, fc, dfc); break;
    case 5: cutoffFdfT<R, 5>(P, g, r, fc, dfc); break;
    case 6: cutoffFdfT<R, 6>(P, g, r, fc, dfc); break;
    case 7: cutoffFdfT<R, 7>(P, g, r, fc, dfc); break;
    default: cutoffFdfT<R, 8>(P, g, r, fc, dfc); break;
    }
}

// pow_int (libnnp/utility.cpp:292-317): exponentiation by squaring.
template <typename R>
__device__ __forceinline__ R powInt(R x, int n)
{
    unsigned m;
    if (n < 0)
    {
        x = R(1) / x;
        m = (unsigned)(-n);
    }
    else m = (unsigned)n;
    R result = R(1);
    do
    {
        if (m & 1u) result *= x;
        m >>= 1;
        x *= x;
    }
    while (m);
    return result;
}

// powInt for 0 <= n < 16 without branches: the same multiplications as
// the loop above for the bits of n (lanes with different exponents do not
// diverge).  Used by the product-form path where it measured faster: the
// 8-shape kernels (zeta up to 16) and FP32.
template <typename R>
__device__ __forceinline__ R powInt16(R x, int n)
{
    R result = R(1);
#pragma unroll
    for (int b = 0; b < 4; ++b)
    {
        R const t = result * x;
        result = ((n >> b) & 1) ? t : result;
        x *= x;
    }
    return result;
}

// Inverse factorials 1 / n! as compile-time constants.
template <int N>
struct InvFact
{
    static constexpr double value = InvFact<N - 1>::value / double(N);
};
template <>
struct InvFact<0>
{
    static constexpr double value = 1.0;
};

// Horner steps n = N .. 0 of sum_n (-1)^n v^n / (2n + K)!  (K = 0: cos,
// K = 1: sin(x) / x, with x^2 = v).
template <int N, int K>
struct AltSeries
{
    __device__ static __forceinline__ double run(double v, double acc)
    {
        constexpr double c = ((N & 1) ? -1.0 : 1.0) * InvFact<2 * N + K>::value;
        return AltSeries<N - 1, K>::run(v, fma(acc, v, c));
    }
};
template <int K>
struct AltSeries<-1, K>
{
    __device__ static __forceinline__ double run(double, double acc)
    {
        return acc;
    }
};

// The cosine cutoff (alpha = 0) of a pair distance r from v = (a r)^2,
// a = pi / rc, without a square root or sin / cos: the Taylor series
//   cos(a r)          = sum_{n>=0} (-1)^n v^n / (2n)!
//   sin(a r) / (a r)  = sum_{n>=0} (-1)^n v^n / (2n + 1)!
// by Horner's rule.  For 0 <= v <= pi^2 (r <= rc) the first omitted terms
// are below 3.1e-18 (cos, n = 16) and 9.4e-18 (sin / x, n = 15).
__device__ __forceinline__ void cosSincSeries(double v, double& c, double& s)
{
    c = AltSeries<15, 0>::run(v, 0.0);
    s = AltSeries<14, 1>::run(v, 0.0);
}

// The same cutoff through the half angle, from w = v / 4 = (a r / 2)^2:
//   ch = cos(a r / 2),  sh = sin(a r / 2) / (a r / 2)
// (Taylor series by Horner's rule, started at the n = 10 coefficient), so
// that f_c = (cos(a r) + 1) / 2 = ch^2 and sin(a r) / (a r) = sh ch.  For
// 0 <= w <= pi^2 / 4 (r <= rc) the first omitted terms are below 1.9e-17
// (cos, n = 11) and 8.1e-19 (sin / x, n = 11): ten FMAs per series
// instead of fifteen, and no cancellation in f_c near rc.
__device__ __forceinline__ void halfAngleCosSinc(double w, double& ch,
                                                 double& sh)
{
    constexpr double c10 = InvFact<20>::value;
    constexpr double s10 = InvFact<21>::value;
    ch = AltSeries<9, 0>::run(w, c10);
    sh = AltSeries<9, 1>::run(w, s10);
}

// Per-warp shared-memory views.
template <typename R>
struct WarpMem
{
    R*        dx;
    R*        dy;
    R*        dz;
    R*        d;
    R*        inv;    // 1 / d
    R*        fc;
    R*        dfcr;   // dfc / d
    R*        E;      // [expIdx][cap]
    unsigned* bits;   // [owner][words]
    double const* expTab;  // the exponential's 2^(j / 64) table (staged
                           // kernel, FP64)
    R*        wpG;    // [maxSF]
    struct Cat*  cats;  // work-item categories of the current segment
    unsigned*    itemList;  // sort mode 4: (category << 16 | owner) items
    int*         itemHist;  // sort mode 4: [cap + 1] count histogram
    int          sortCats;  // bit 0: order angular categories by partner
                            // count; bit 1: balanced owner order; bit 2:
                            // one item list of the segment ordered by
                            // partner count (buildItemList)
    // The categories are followed (kCatsBytes further on) by the balanced
    // owner order: the owners of each element ordered by their number of
    // valid partners of element e2 (descending in 32 count buckets, ties by
    // position), order[e2 * cap + t] for t in the owner element's range,
    // then 32 ints of sort scratch.  The narrow angular paths walk owners
    // in that order so that the 32 owners of a round have similar loop
    // lengths.
};

// A category is a group together with one owner element: its items are the
// owners t in [ob, ob + on) and each iterates partners in [pb, pe).
struct Cat
{
    int gi, et, ob, on, pb, pe;
    int oo;   // offset of the owners in the balanced order, -1: positions
};
// Segments hold at most kMaxSegGroups groups (longer runs of equal (type, rc)
// are split), so the category table never overflows.
constexpr int kMaxSegGroups = 16;
constexpr int kMaxCats = 2 * kMaxSegGroups;
// Groups per segment: element-weighted groups give one category per owner
// element, the others at most two.
__host__ __device__ constexpr int segCap(int type)
{
    return (type == 12 || type == 13 || type >= 23) ? kMaxCats / kMaxElem
                                                    : kMaxSegGroups;
}
constexpr long kCatsBytes = ((long)(kMaxCats * sizeof(Cat)) + 15) / 16 * 16;

// The balanced owner order and its sort scratch (see WarpMem).
template <typename R>
__device__ __forceinline__ unsigned short* ownerOrder(WarpMem<R> const& W)
{
    return reinterpret_cast<unsigned short*>(
        reinterpret_cast<char*>(W.cats) + kCatsBytes);
}

// Items the sort-mode-4 list holds per neighbor of the atom (a segment of
// groups with two owner sides per group pair has up to 2 x groups x
// neighbors items; more fall back to positional order).
constexpr int kItemsPerCap = 4;

// Bytes of one warp's shared-memory region (16-byte multiple).
template <typename R>
__host__ __device__ inline long warpBytes(int maxExp, int maxSF, int cap,
                                          int numElements)
{
    long const words = (cap + 31) / 32;
    long b = (long)sizeof(R) * (7L * cap + (long)maxExp * cap + maxSF);
    b = (b + 15) / 16 * 16;
    b += 4L * cap * words;                          // validity bits
    b = (b + 15) / 16 * 16;
    b += kCatsBytes;                                // categories
    b += (2L * numElements * cap + 3) / 4 * 4;      // owner order
    b += 4L * 32;                                   // count buckets
    b += 4L * kItemsPerCap * cap;                   // item list
    b += 4L * (cap + 2);                            // its count histogram
    return (b + 15) / 16 * 16;
}

// Offset of the item list behind the categories (the layout above).
__host__ __device__ inline long itemListOffset(int cap, int numElements)
{
    return kCatsBytes + (2L * numElements * cap + 3) / 4 * 4 + 4L * 32;
}

// Adds each lane's G contribution for symmetry function `sf` (-1 =
// nothing) into the warp sums.  `key` identifies the lane's work-item
// category; lanes of one category occupy contiguous lanes (items are
// enumerated category by category).  One segmented butterfly reduces every
// run at once in a fixed lane order; the runs' first lanes then add their
// totals one after another (two runs may share sf).
template <typename R>
__device__ __forceinline__ void flushBySF(WarpMem<R> const& W, int key, int sf,
                                          R g)
{
    int const lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        R const a = __shfl_down_sync(kFull, g, off);
        int const ko = __shfl_down_sync(kFull, key, off);
        if (lane + off < 32 && ko == key) g += a;
    }
    int const prev = __shfl_up_sync(kFull, key, 1);
    bool const head = (lane == 0) || (prev != key);
    unsigned heads = __ballot_sync(kFull, head && sf >= 0);
    while (heads)
    {
        if (lane == __ffs(heads) - 1) W.wpG[sf] += g;
        __syncwarp();
        heads &= heads - 1;
    }
}

struct Item
{
    int gi;      // group index, -1 = no item
    int key;     // category index, -1 = no item
    int t;       // owner neighbor position
    int et;      // owner element
    int pb, pe;  // partner range
};

// Builds the categories of segment [g0, g1) into W.cats (lane 0) and
// returns the number of items.  Angular categories are ordered by partner
// count, largest first (stable), so that the lanes of a round have similar
// trip counts.
template <typename R>
__device__ __forceinline__ int buildCats(DevGroup const* G, int g0, int g1,
                                         int const eb[kMaxElem + 1],
                                         bool byPartners, int orderCap,
                                         WarpMem<R> const& W, int& ncat)
{
    int const lane = threadIdx.x & 31;
    int n = 0, total = 0;
    if (lane == 0)
    {
        for (int gi = g0; gi < g1; ++gi)
        {
            DevGroup const& g = G[gi];
            if (g.type == 12 || g.type == 13 || g.type >= 23)
            {
                // Element-weighted groups: owners of every element,
                // partners of every element.
                for (int et = 0; et < kMaxElem; ++et)
                {
                    if (eb[et + 1] <= eb[et]) continue;
                    Cat c;
                    c.gi = gi;
                    c.et = et;
                    c.ob = eb[et];
                    c.on = eb[et + 1] - eb[et];
                    c.pb = 0;
                    c.pe = eb[kMaxElem];
                    c.oo = -1;
                    W.cats[n++] = c;
                    total += c.on;
                }
                continue;
            }
            bool const radial = (g.type == 2 || g.type == 20);
            int const sides = (radial || g.e1 == g.e2) ? 1 : 2;
            for (int sd = 0; sd < sides; ++sd)
            {
                int const et = (sd == 0) ? g.e1 : g.e2;
                int const pe2 = radial ? g.e1
                              : ((sd == 0) ? g.e2 : g.e1);
                Cat c;
                c.gi = gi;
                c.et = et;
                c.ob = eb[et];
                c.on = eb[et + 1] - eb[et];
                c.pb = eb[pe2];
                c.pe = eb[pe2 + 1];
                c.oo = orderCap > 0 ? pe2 * orderCap + c.ob : -1;
                int pos = n;
                if (byPartners)
                    while (pos > 0 && (W.cats[pos - 1].pe - W.cats[pos - 1].pb)
                                          < (c.pe - c.pb))
                    {
                        W.cats[pos] = W.cats[pos - 1];
                        --pos;
                    }
                W.cats[pos] = c;
                ++n;
                total += c.on;
            }
        }
    }
    ncat = __shfl_sync(kFull, n, 0);
    total = __shfl_sync(kFull, total, 0);
    __syncwarp();
    return total;
}

template <typename R>
__device__ __forceinline__ Item itemOf(WarpMem<R> const& W, int ncat, int q)
{
    Item it;
    it.gi = -1;
    it.key = -1;
    it.t = 0;
    it.et = 0;
    it.pb = it.pe = 0;
    for (int c = 0; c < ncat; ++c)
    {
        Cat const cc = W.cats[c];
        if (q < cc.on)
        {
            it.gi = cc.gi;
            it.key = c;
            it.t = cc.oo >= 0 ? (int)ownerOrder(W)[cc.oo + q] : cc.ob + q;
            it.et = cc.et;
            it.pb = cc.pb;
            it.pe = cc.pe;
            return it;
        }
        q -= cc.on;
    }
    return it;
}

// Partner mask of word w restricted to [pb, pe).
__device__ __forceinline__ unsigned rangeMask(unsigned m, int w, int pb,
                                              int pe);

// Sort mode 4 (narrow angular segments): the segment's work items
// (category, owner) as one list, ordered by the owner's number of valid
// partners (descending; ties in item order, so the order is deterministic)
// and, inside every round of 32, by category -- flushBySF needs the lanes
// of a category contiguous, and a round's trip count is its largest
// partner count, so rounds of similar counts keep the lanes busy across
// the categories (positional or per-category order leaves about a third
// of the lane-iterations idle on water).  Returns false when the segment
// has more items than the list holds (the caller keeps positional order).
template <typename R>
__device__ bool buildItemList(WarpMem<R> const& W, int ncat, int items,
                              int words, int cap)
{
    int const lane = threadIdx.x & 31;
    if (items > kItemsPerCap * cap) return false;
    auto itemAt = [&](int q, int& c, int& t) {
        c = 0;
        while (c < ncat - 1 && q >= W.cats[c].on)
        {
            q -= W.cats[c].on;
            ++c;
        }
        t = W.cats[c].ob + q;
    };
    auto countOf = [&](int c, int t) {
        Cat const& cc = W.cats[c];
        int n = 0;
        for (int w = cc.pb >> 5; w < (cc.pe + 31) >> 5; ++w)
            n += __popc(rangeMask(W.bits[t * words + w], w, cc.pb, cc.pe));
        return min(n, cap);
    };
    int* const hist = W.itemHist;
    for (int k = lane; k <= cap; k += 32) hist[k] = 0;
    __syncwarp();
    for (int q = lane; q < items; q += 32)
    {
        int c, t;
        itemAt(q, c, t);
        atomicAdd(&hist[countOf(c, t)], 1);
    }
    __syncwarp();
    if (lane == 0)
    {
        // hist[n] := first position of count n (descending counts).
        int run = 0;
        for (int k = cap; k >= 0; --k)
        {
            int const h = hist[k];
            hist[k] = run;
            run += h;
        }
    }
    __syncwarp();
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        int const q = q0 + lane;
        bool const act = q < items;
        int c = 0, t = 0, n = -1 - lane;
        if (act)
        {
            itemAt(q, c, t);
            n = countOf(c, t);
        }
        unsigned const peers = __match_any_sync(kFull, n);
        int const r = __popc(peers & ((1u << lane) - 1u));
        if (act)
            W.itemList[hist[n] + r] = ((unsigned)c << 16) | (unsigned)t;
        __syncwarp();
        if (act && r == 0) hist[n] += __popc(peers);
        __syncwarp();
    }
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        int const q = q0 + lane;
        unsigned const v = q < items ? W.itemList[q] : 0xffffffffu;
        int const key = q < items ? (int)(v >> 16) : 0x7fffffff;
        int rank = 0;
        for (int o = 0; o < 32; ++o)
        {
            int const ko = __shfl_sync(kFull, key, o);
            rank += (ko < key || (ko == key && o < lane)) ? 1 : 0;
        }
        __syncwarp();
        if (q < items) W.itemList[q0 + rank] = v;
        __syncwarp();
    }
    return true;
}

template <typename R>
__device__ __forceinline__ Item itemFromList(WarpMem<R> const& W, int items,
                                             int q)
{
    Item it;
    it.gi = -1;
    it.key = -1;
    it.t = 0;
    it.et = 0;
    it.pb = it.pe = 0;
    if (q >= items) return it;
    unsigned const v = W.itemList[q];
    Cat const cc = W.cats[v >> 16];
    it.gi = cc.gi;
    it.key = (int)(v >> 16);
    it.t = (int)(v & 0xffffu);
    it.et = cc.et;
    it.pb = cc.pb;
    it.pe = cc.pe;
    return it;
}

// Partner mask of word w restricted to [pb, pe).
__device__ __forceinline__ unsigned rangeMask(unsigned m, int w, int pb,
                                              int pe)
{
    int const base = w << 5;
    if (base < pb) m &= kFull << (pb - base);
    if (base + 32 > pe)
    {
        int const keep = pe - base;
        m &= (keep >= 32) ? kFull : ((1u << keep) - 1u);
    }
    return m;
}

// Balanced owner order for owners [ob, oe) and partners [pb, pe): the owners
// sorted by their number of valid partners, descending, by a stable warp
// counting sort over 32 buckets of the count range (exact when the counts
// span at most 32 values). Writes order[ob .. oe). Warp-uniform arguments.
// The counts of the first kOrderCached rounds of 32 owners are kept in
// registers across the three passes (min / max, histogram, placement);
// later rounds count again.
constexpr int kOrderCached = 4;
template <typename R>
__device__ void buildOwnerOrder(WarpMem<R> const& W, int words, int ob,
                                int oe, int pb, int pe,
                                unsigned short* __restrict__ order,
                                int* __restrict__ hist)
{
    int const lane = threadIdx.x & 31;
    if (oe <= ob) return;
    auto count = [&](int t) {
        int c = 0;
        for (int w = pb >> 5; w < (pe + 31) >> 5; ++w)
            c += __popc(rangeMask(W.bits[t * words + w], w, pb, pe));
        return c;
    };
    int cc[kOrderCached];
    int cmin = 0x7fffffff, cmax = 0;
#pragma unroll
    for (int r = 0; r < kOrderCached; ++r)
    {
        int const t = ob + 32 * r + lane;
        cc[r] = (t < oe) ? count(t) : 0;
        if (t < oe)
        {
            cmin = min(cmin, cc[r]);
            cmax = max(cmax, cc[r]);
        }
    }
    for (int t = ob + 32 * kOrderCached + lane; t < oe; t += 32)
    {
        int const c = count(t);
        cmin = min(cmin, c);
        cmax = max(cmax, c);
    }
    for (int o = 16; o > 0; o >>= 1)
    {
        cmin = min(cmin, __shfl_xor_sync(kFull, cmin, o));
        cmax = max(cmax, __shfl_xor_sync(kFull, cmax, o));
    }
    int const span = cmax - cmin + 1;
    // Bucket 0 holds the owners with the most partners.
    auto key = [&](int c) { return ((cmax - c) * 32) / span; };
    hist[lane] = 0;
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kOrderCached; ++r)
        if (ob + 32 * r + lane < oe) atomicAdd(&hist[key(cc[r])], 1);
    for (int t = ob + 32 * kOrderCached + lane; t < oe; t += 32)
        atomicAdd(&hist[key(count(t))], 1);
    __syncwarp();
    int const h = hist[lane];
    int incl = h;
    for (int o = 1; o < 32; o <<= 1)
    {
        int const v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += v;
    }
    __syncwarp();
    hist[lane] = incl - h;
    __syncwarp();
    auto place = [&](int t0, int c) {
        int const t = t0 + lane;
        bool const active = t < oe;
        int const k = active ? key(c) : 32 + lane;
        unsigned const peers = __match_any_sync(kFull, k);
        int const r = __popc(peers & ((1u << lane) - 1u));
        if (active) order[ob + hist[k] + r] = (unsigned short)t;
        __syncwarp();
        if (active && r == 0) hist[k] += __popc(peers);
        __syncwarp();
    };
#pragma unroll
    for (int r = 0; r < kOrderCached; ++r)
        if (ob + 32 * r < oe) place(ob + 32 * r, cc[r]);
    for (int t0 = ob + 32 * kOrderCached; t0 < oe; t0 += 32)
        place(t0, t0 + lane < oe ? count(t0 + lane) : 0);
}

// Rounds of 32 owners start at qBegin and advance by qStep (several warps
// of one atom split the owners: warp w takes qBegin = 32 w, qStep = 32 x
// warps).
template <typename R, int MC>
__device__ void radialSegment(SFParams const& P, DevGroup const* G,
                              DevMember const* M, int g0, int g1,
                              int const eb[kMaxElem + 1], int cnt,
                              WarpMem<R> const& W, R* __restrict__ out,
                              int derivatives, int qBegin = 0,
                              int qStep = 32)
{
    int const lane = threadIdx.x & 31;
    int ncat = 0;
    int const items = buildCats(G, g0, g1, eb, false, 0, W, ncat);
    int maxM = 0;
    for (int gi = g0; gi < g1; ++gi) maxM = max(maxM, G[gi].mcnt);
    for (int q0 = qBegin; q0 < items; q0 += qStep)
    {
        Item const it = itemOf(W, ncat, q0 + lane);
        bool const active = it.gi >= 0;
        DevGroup const& g = G[active ? it.gi : g0];
        int const t = it.t;
        R const r = W.d[t];
        bool const valid = active && (r < R(g.rc));
        R const pfc = W.fc[t], pdfcr = W.dfcr[t], inv = W.inv[t];
        R const d1[3] = {W.dx[t], W.dy[t], W.dz[t]};
        // SymGrpExpRadWeighted (type 12): weight = atomic number of j.
        R const z = (g.type == 12) ? R(P.atomicNumber[it.et]) : R(1);
        for (int mb = 0; mb < maxM; mb += MC)
        {
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                bool const has = active && (mb + l < g.mcnt);
                DevMember const& m = M[g.mbeg + (has ? mb + l : 0)];
                R gs = R(0), p1 = R(0);
                if (has && valid)
                {
                    // SymGrpExpRad.cpp:210-211 with (f_c' - 2 eta (r - rs) f_c)/r
                    // written as f_c'/r - 2 eta (r - rs) f_c / r.
                    R const eta = R(m.eta);
                    R const rr = r - R(m.rs);
                    R const pexp = z * mexp(-eta * rr * rr);
                    gs = pexp * pfc;
                    p1 = R(m.factorNorm)
                       * (pdfcr - R(2) * eta * rr * pfc * inv) * pexp;
                }
                R const sx = p1 * d1[0], sy = p1 * d1[1], sz = p1 * d1[2];
                if (derivatives && has)
                {
                    long const s = m.slot[it.et];
                    out[(s * 3 + 0) * cnt + t] = -sx;
                    out[(s * 3 + 1) * cnt + t] = -sy;
                    out[(s * 3 + 2) * cnt + t] = -sz;
                }
                flushBySF(W, it.key, has ? (int)m.sf : -1, gs);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Compact symmetry functions (types 20, 21, 22).
// ---------------------------------------------------------------------------

// CoreFunction::fdf for the compact core functions (libnnp/CoreFunction.h:
// 171-320; POLY1..4 and EXP, the subtypes SymFncBaseComp accepts).
template <typename R>
__device__ __forceinline__ void coreFdf(int core, R x, R E, R& fx, R& dfx)
{
    if (core == CC_EXP)
    {
        R const temp = R(1) / (x * x - R(1));
        R const temp2 = mexp(temp);
        fx = E * temp2;
        dfx = R(-2) * E * x * temp * temp * temp2;
    }
    else if (core == CC_POLY1)
    {
        fx = (R(2) * x - R(3)) * x * x + R(1);
        dfx = x * (R(6) * x - R(6));
    }
    else if (core == CC_POLY2)
    {
        R const x2 = x * x;
        fx = ((R(15) - R(6) * x) * x - R(10)) * x * x2 + R(1);
        dfx = x2 * ((R(60) - R(30) * x) * x - R(30));
    }
    else if (core == CC_POLY3)
    {
        R const x2 = x * x;
        fx = (x * (x * (R(20) * x - R(70)) + R(84)) - R(35)) * x2 * x2 + R(1);
        dfx = x2 * x * (x * (x * (R(140) * x - R(420)) + R(420)) - R(140));
    }
    else
    {
        R x4 = x * x;
        x4 *= x4;
        fx = (x * (x * ((R(315) - R(70) * x) * x - R(540)) + R(420))
              - R(126)) * x * x4 + R(1);
        dfx = x4 * (x * (x * ((R(2520) - R(630) * x) * x - R(3780))
                         + R(2520)) - R(630));
    }
}

// CompactFunction::fdf (libnnp/CompactFunction.h:160-167) with
// CoreFunction's asymmetric variant x -> (2 - x) x.
template <typename R>
__device__ __forceinline__ void compactFdf(int core, bool asym, R center,
                                           R scale, R a, R E, R& f, R& df)
{
    R const u = (a - center) * scale;
    R const x = u < R(0) ? -u : u;
    R fx, dfx;
    if (asym)
    {
        coreFdf<R>(core, (R(2) - x) * x, E, fx, dfx);
        dfx *= R(2) - R(2) * x;
    }
    else coreFdf<R>(core, x, E, fx, dfx);
    f = fx;
    df = dfx * (u < R(0) ? -scale : scale);
}

// SymGrpCompRad::calculate (libnnp/SymGrpCompRad.cpp:142-219): work items
// (group, neighbor j of element e1); G_m = sum_j f_m(r_ij) over
// rl_m < r_ij < rc_m, slot_m(j) = -sf_m f_m'(r_ij) / r_ij dr_ij.
template <typename R, int MC>
__device__ void compactRadialSegment(SFParams const& P, DevGroup const* G,
                                     DevMember const* M, int g0, int g1,
                                     int const eb[kMaxElem + 1], int cnt,
                                     WarpMem<R> const& W, R* __restrict__ out,
                                     int derivatives)
{
    int const lane = threadIdx.x & 31;
    int ncat = 0;
    int const items = buildCats(G, g0, g1, eb, false, 0, W, ncat);
    int maxM = 0;
    for (int gi = g0; gi < g1; ++gi) maxM = max(maxM, G[gi].mcnt);
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        Item const it = itemOf(W, ncat, q0 + lane);
        bool const active = it.gi >= 0;
        DevGroup const& g = G[active ? it.gi : g0];
        int const t = it.t;
        R const r = W.d[t];
        bool const valid = active && (r < R(g.rc)) && (r > R(0));
        R const d1[3] = {W.dx[t], W.dy[t], W.dz[t]};
        // SymGrpCompRadWeighted (type 23): weight = atomic number of j.
        R const z = (g.type == 23) ? R(P.atomicNumber[it.et]) : R(1);
        for (int mb = 0; mb < maxM; mb += MC)
        {
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                bool const has = active && (mb + l < g.mcnt);
                DevMember const& m = M[g.mbeg + (has ? mb + l : 0)];
                R gs = R(0), p1 = R(0);
                if (has && valid && r > R(m.eta) && r < R(m.rs))
                {
                    R rad, drad;
                    compactFdf<R>(m.zetaInt, m.useIntPow != 0,
                                  R(m.factorDeriv), R(m.zetaLambda), r,
                                  R(P.E), rad, drad);
                    gs = z * rad;
                    p1 = drad * (z * R(m.factorNorm) / r);
                }
                if (derivatives && has)
                {
                    long const s = m.slot[it.et];
                    out[(s * 3 + 0) * cnt + t] = -(p1 * d1[0]);
                    out[(s * 3 + 1) * cnt + t] = -(p1 * d1[1]);
                    out[(s * 3 + 2) * cnt + t] = -(p1 * d1[2]);
                }
                flushBySF(W, it.key, has ? (int)m.sf : -1, gs);
            }
        }
    }
}

// SymGrpCompAngn::calculate / SymGrpCompAngw::calculate
// (libnnp/SymGrpCompAngn.cpp:171-383, SymGrpCompAngw.cpp) in owner-computes
// form: the owner j of an item visits every partner k of the other element;
// per member, with the reference's open-interval tests on r_ij, r_ik, r_jk
// (narrow) and the angle theta = acos(cos theta_ijk),
//   term = f(r_ij) f(r_ik) [f(r_jk)] g(theta),
//   p_own = sf (rad phi_own g' acos' + g chi_own),  p3 = sf (rad psi g' acos'
//   + g chi_jk), slot(j) = -(sum_k p_own dr_ij + p3 (dr_ik - dr_ij)),
// the reference's p1 (owner first) or p2 (owner second).  The reference
// reuses f(r_jk) of the previous member when calculateComp is false and
// that member was not skipped; the source member is found by walking back
// over the run (same rl, rc: only the angle test can differ).  A radial
// value that underflows to zero inside its support skips the member here
// whichever neighbor comes first; the reference checks the first one only,
// which changes nothing but that reuse chain.  Narrow groups walk the
// per-atom validity bitmask built with rc = rmax (the reference's group-level
// r_ik < rmax, r_jk^2 < rmax^2 tests); the owner's radial values are formed
// once per item and the partner's once per radial function id.
template <typename R, int MC, bool NARROW>
__device__ void compactAngularSegment(SFParams const& P, DevGroup const* G,
                                      DevMember const* M, int g0, int g1,
                                      int const eb[kMaxElem + 1], int cnt,
                                      int words, WarpMem<R> const& W,
                                      R* __restrict__ out, int derivatives)
{
    int const lane = threadIdx.x & 31;
    int ncat = 0;
    int const items = buildCats(G, g0, g1, eb, false, 0, W, ncat);
    int maxM = 0;
    for (int gi = g0; gi < g1; ++gi) maxM = max(maxM, G[gi].mcnt);
    R const E = R(P.E);
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        Item const it = itemOf(W, ncat, q0 + lane);
        bool const active = it.gi >= 0;
        DevGroup const& g = G[active ? it.gi : g0];
        int const t = it.t;
        R const rij = W.d[t];
        R const rmax = R(g.rc);
        bool const valid = active && (rij < rmax) && (rij > R(0));
        R const dr1[3] = {W.dx[t], W.dy[t], W.dz[t]};
        for (int mb = 0; mb < maxM; mb += MC)
        {
            int const mc = active ? min(MC, g.mcnt - mb) : 0;
            R aG[MC], aP[MC], aQx[MC], aQy[MC], aQz[MC];
            // The owner's radial value per member (0: r_ij outside).
            R radO[MC], dradO[MC];
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                aG[l] = aP[l] = aQx[l] = aQy[l] = aQz[l] = R(0);
                radO[l] = dradO[l] = R(0);
                if (l < mc)
                {
                    DevMember const& mm = M[g.mbeg + mb + l];
                    if (rij > R(mm.eta) && rij < R(mm.rs))
                        compactFdf<R>(mm.zetaInt, mm.useIntPow != 0,
                                      R(mm.factorDeriv), R(mm.zetaLambda),
                                      rij, E, radO[l], dradO[l]);
                }
            }
            if (valid && mc > 0)
            {
                // Partners: the narrow validity bitmask (r_ik < rmax,
                // r_jk^2 < rmax^2), or every k of the partner element.
                int const wb = it.pb >> 5;
                int const we = (it.pe + 31) >> 5;
                int w = wb - 1;
                unsigned m = 0u;
                for (;;)
                {
                    while (m == 0u && ++w < we)
                        m = rangeMask(NARROW ? W.bits[t * words + w] : kFull,
                                      w, it.pb, it.pe);
                    if (m == 0u) break;
                    int const k = (w << 5) + __ffs(m) - 1;
                    m &= m - 1;
                    R const rik = W.d[k];
                    if (!NARROW && (k == t || !(rik < rmax))) continue;
                    R const dr2[3] = {W.dx[k], W.dy[k], W.dz[k]};
                    R const dr3[3] = {dr2[0] - dr1[0], dr2[1] - dr1[1],
                                      dr2[2] - dr1[2]};
                    R rjk = R(0), rinvjk = R(0);
                    if (NARROW)
                    {
                        R const r2 = dr3[0] * dr3[0] + dr3[1] * dr3[1]
                                   + dr3[2] * dr3[2];
                        if (r2 <= R(0)) continue;
                        rjk = sqrt(r2);
                        rinvjk = R(1) / rjk;
                    }
                    R const rinvijik = R(1) / (rij * rik);
                    R const costijk = (dr1[0] * dr2[0] + dr1[1] * dr2[1]
                                       + dr1[2] * dr2[2]) * rinvijik;
                    if (costijk <= R(-1) || costijk >= R(1)) continue;
                    R const theta = acos(costijk);
                    R const rinvOwn = rinvijik * rik;
                    R const rinvPart = rinvijik * rij;
                    R const phi0 = rinvOwn * (rinvPart - rinvOwn * costijk);
                    R const dacos = derivatives
                        ? R(-1) / sqrt(R(1) - costijk * costijk) : R(0);
                    // SymGrpCompAng[nw]Weighted (types 24, 25): weight
                    // Z_j Z_k on the term and its derivatives.
                    R zz = R(1);
                    if (g.type >= 24)
                    {
                        int ek = 0;
                        while (k >= eb[ek + 1]) ++ek;
                        zz = R(P.atomicNumber[it.et] * P.atomicNumber[ek]);
                    }
                    // Radial values of the partner (and of r_jk) for the
                    // current radial function id.
                    int rid = -1;
                    R radP = R(0), dradP = R(0), radJ = R(0), dradJ = R(0);
#pragma unroll
                    for (int l = 0; l < MC; ++l)
                    {
                        if (l >= mc) break;
                        int const mi = mb + l;
                        DevMember const& mm = M[g.mbeg + mi];
                        R const rl = R(mm.eta), rc = R(mm.rs);
                        if (radO[l] == R(0) || rik <= rl || rik >= rc
                            || (NARROW && (rjk <= rl || rjk >= rc))
                            || theta <= R(mm.lambda) || theta >= R(mm.zeta))
                            continue;
                        int const core = mm.zetaInt;
                        bool const asym = mm.useIntPow != 0;
                        R const c0 = R(mm.factorDeriv), c1 = R(mm.zetaLambda);
                        if ((int)mm.rsPositive != rid)
                        {
                            rid = mm.rsPositive;
                            compactFdf<R>(core, asym, c0, c1, rik, E, radP,
                                          dradP);
                            if (NARROW)
                                compactFdf<R>(core, asym, c0, c1, rjk, E,
                                              radJ, dradJ);
                        }
                        if (radP == R(0)) continue;
                        R radjk = R(1), dradjk = R(0);
                        if (NARROW)
                        {
                            radjk = radJ;
                            dradjk = dradJ;
                            int src = mi;
                            while (src > 0 && !M[g.mbeg + src].calcExp
                                   && theta > R(M[g.mbeg + src - 1].lambda)
                                   && theta < R(M[g.mbeg + src - 1].zeta))
                                --src;
                            DevMember const& ms = M[g.mbeg + src];
                            if (ms.rsPositive != mm.rsPositive)
                                compactFdf<R>(ms.zetaInt, ms.useIntPow != 0,
                                              R(ms.factorDeriv),
                                              R(ms.zetaLambda), rjk, E,
                                              radjk, dradjk);
                        }
                        R ang, dang;
                        compactFdf<R>(core, false, R(mm.aCenter),
                                      R(mm.aScale), theta, E, ang, dang);
                        ang *= zz;
                        dang *= zz;
                        R const rad = radO[l] * radP * radjk;
                        aG[l] += rad * ang;
                        if (!derivatives) continue;
                        dang *= dacos;
                        R const sf = R(mm.factorNorm);
                        R const chiOwn = rinvOwn * dradO[l] * radP * radjk;
                        R const pOwn = (sf * rad) * (phi0 * dang)
                                     + (sf * ang) * chiOwn;
                        R p3 = (sf * rad) * (rinvijik * dang);
                        if (NARROW)
                            p3 += (sf * ang) * (-rinvjk * radO[l] * radP
                                                * dradjk);
                        aP[l] += pOwn;
                        aQx[l] += p3 * dr3[0];
                        aQy[l] += p3 * dr3[1];
                        aQz[l] += p3 * dr3[2];
                    }
                }
            }
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                bool const has = l < mc;
                DevMember const& mm = M[g.mbeg + (has ? mb + l : 0)];
                if (derivatives && has)
                {
                    long const s = mm.slot[it.et];
                    out[(s * 3 + 0) * cnt + t] = -(aP[l] * dr1[0] + aQx[l]);
                    out[(s * 3 + 1) * cnt + t] = -(aP[l] * dr1[1] + aQy[l]);
                    out[(s * 3 + 2) * cnt + t] = -(aP[l] * dr1[2] + aQz[l]);
                }
                flushBySF(W, it.key, has ? (int)mm.sf : -1, R(0.5) * aG[l]);
            }
        }
    }
}

// General angular path: the reference's per-member expression form.
template <typename R, int CT, int MC, bool NARROW>
__device__ void angularGeneric(SFParams const& P, DevGroup const* G,
                               DevMember const* M, int g0, int g1,
                               int const eb[kMaxElem + 1], int cnt, int words,
                               int capE, WarpMem<R> const& W,
                               R* __restrict__ out, int derivatives)
{
    int const lane = threadIdx.x & 31;
    int ncat = 0;
    int const items = buildCats(G, g0, g1, eb, (W.sortCats & 1) != 0,
                                (NARROW && (W.sortCats & 2)) ? capE : 0, W,
                                ncat);
    int maxM = 0;
    for (int gi = g0; gi < g1; ++gi) maxM = max(maxM, G[gi].mcnt);
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        Item const it = itemOf(W, ncat, q0 + lane);
        bool const active = it.gi >= 0;
        DevGroup const& g = G[active ? it.gi : g0];
        int const t = it.t;
        R const rij = W.d[t];
        R const rc = R(g.rc);
        bool const valid = active && (rij < rc);
        R const dr1[3] = {W.dx[t], W.dy[t], W.dz[t]};
        R const invij = W.inv[t];
        R const pfcij = W.fc[t];
        R const pdfcrij = W.dfcr[t];
        for (int mb = 0; mb < maxM; mb += MC)
        {
            int const mc = active ? min(MC, g.mcnt - mb) : 0;
            R aG[MC], aP1[MC], aPx[MC], aPy[MC], aPz[MC];
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                aG[l] = R(0);
                aP1[l] = R(0);
                aPx[l] = R(0);
                aPy[l] = R(0);
                aPz[l] = R(0);
            }
            if (valid && mc > 0)
            {
                R const cr0 = invij * invij;  // 1 / r_ij^2
                int const wb = it.pb >> 5;
                int const we = (it.pe + 31) >> 5;
                // One loop over the lane's partners (not one per mask
                // word): the warp's trip count is the largest partner count
                // of its lanes, not the sum of per-word maxima.
                int w = wb - 1;
                unsigned m = 0u;
                for (;;)
                {
                    while (m == 0u && ++w < we)
                        m = rangeMask(NARROW ? W.bits[t * words + w] : kFull,
                                      w, it.pb, it.pe);
                    if (m == 0u) break;
                    {
                        int const k = (w << 5) + __ffs(m) - 1;
                        m &= m - 1;
                        if (!NARROW)
                        {
                            if (k == t || !(W.d[k] < rc)) continue;
                        }
                        R const dr2[3] = {W.dx[k], W.dy[k], W.dz[k]};
                        R const dr3[3] = {dr2[0] - dr1[0], dr2[1] - dr1[1],
                                          dr2[2] - dr1[2]};
                        R const invik = W.inv[k];
                        R const pfcik = W.fc[k];
                        R const rinvijik = invij * invik;
                        R const costijk = (dr1[0] * dr2[0] + dr1[1] * dr2[1]
                                           + dr1[2] * dr2[2]) * rinvijik;
                        R const cr = costijk * cr0;
                        R rjk = R(0), invjk = R(0), pfcjk = R(1),
                          pdfcjk = R(0);
                        if (NARROW)
                        {
                            R const r2 = dr3[0] * dr3[0] + dr3[1] * dr3[1]
                                       + dr3[2] * dr3[2];
                            invjk = mrsqrt(r2);
                            rjk = r2 * invjk;
                            cutoffFdf<R, CT>(P, g, rjk, pfcjk, pdfcjk);
                        }
                        R pfc, pr1, pr3 = R(0);
                        if (NARROW)
                        {
                            pfc = pfcij * pfcik * pfcjk;
                            pr1 = pfcik * pfcjk * pdfcrij;
                            pr3 = pfcij * pfcik * pdfcjk * invjk;
                        }
                        else
                        {
                            pfc = pfcij * pfcik;
                            pr1 = pfcik * pdfcrij;
                        }
                        if (NARROW && g.type == 13)
                        {
                            // SymGrpExpAngnWeighted: weight Z_j Z_k.
                            int ek = 0;
                            while (k >= eb[ek + 1]) ++ek;
                            R const z = R(P.atomicNumber[it.et]
                                          * P.atomicNumber[ek]);
                            pfc *= z;
                            pr1 *= z;
                            pr3 *= z;
                        }
                        R vexp = R(0);
#pragma unroll
                        for (int l = 0; l < MC; ++l)
                        {
                            if (l >= mc) break;
                            DevMember const& mm = M[g.mbeg + mb + l];
                            if (mm.calcExp || l == 0)
                            {
                                R const* E = W.E + (long)mm.expIdx * capE;
                                vexp = E[t] * E[k];
                                if (NARROW)
                                {
                                    R const rjks = rjk - R(mm.rs);
                                    vexp *= mexp(-R(mm.eta) * rjks * rjks);
                                }
                            }
                            R const plambda = R(1) + R(mm.lambda) * costijk;
                            R fg = vexp;
                            if (plambda <= R(0)) fg = R(0);
                            else if (mm.useIntPow)
                                fg *= powInt(plambda, mm.zetaInt - 1);
                            else
                                fg *= mpow(plambda, R(mm.zeta) - R(1));
                            aG[l] += fg * plambda * pfc;
                            fg *= R(mm.factorNorm);
                            R const pfczl = pfc * R(mm.zetaLambda);
                            R const p2etapl = plambda * R(mm.factorDeriv);
                            R p1, p3;
                            if (mm.rsPositive)
                            {
                                R const rijs = rij - R(mm.rs);
                                p1 = fg * (pfczl * (rinvijik - cr
                                                    - p2etapl * rijs * invij)
                                           + pr1 * plambda);
                                if (NARROW)
                                {
                                    R const rjks = rjk - R(mm.rs);
                                    p3 = fg * (pfczl * (rinvijik
                                                        + p2etapl * rjks * invjk)
                                               - pr3 * plambda);
                                }
                                else p3 = fg * pfczl * rinvijik;
                            }
                            else
                            {
                                p1 = fg * (pfczl * (rinvijik - cr - p2etapl)
                                           + pr1 * plambda);
                                if (NARROW)
                                    p3 = fg * (pfczl * (rinvijik + p2etapl)
                                               - pr3 * plambda);
                                else p3 = fg * pfczl * rinvijik;
                            }
                            aP1[l] += p1;
                            aPx[l] += p3 * dr3[0];
                            aPy[l] += p3 * dr3[1];
                            aPz[l] += p3 * dr3[2];
                        }
                    }
                }
            }
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                bool const has = l < mc;
                DevMember const& mm = M[g.mbeg + (has ? mb + l : 0)];
                R const sx = aP1[l] * dr1[0];
                R const sy = aP1[l] * dr1[1];
                R const sz = aP1[l] * dr1[2];
                if (derivatives && has)
                {
                    long const s = mm.slot[it.et];
                    out[(s * 3 + 0) * cnt + t] = -(sx + aPx[l]);
                    out[(s * 3 + 1) * cnt + t] = -(sy + aPy[l]);
                    out[(s * 3 + 2) * cnt + t] = -(sz + aPz[l]);
                }
                flushBySF(W, it.key, has ? (int)mm.sf : -1, R(0.5) * aG[l]);
            }
        }
    }
}

// Product-form angular path (see the header comment): NS shapes per eta
// run, NRC runs per register chunk.
template <typename R, int CT, int NS, int NRC, bool NARROW, bool PIPE>
__device__ void angularFast(SFParams const& P, DevGroup const* G,
                            DevMember const* M, int g0, int g1,
                            int const eb[kMaxElem + 1], int cnt, int words,
                            int capE, WarpMem<R> const& W,
                            R* __restrict__ out, int derivatives)
{
    int const lane = threadIdx.x & 31;
    int ncat = 0;
    bool const global = NARROW && (W.sortCats & 4);
    int const items = buildCats(G, g0, g1, eb,
                                (W.sortCats & 1) != 0 && !global,
                                (NARROW && (W.sortCats & 2) && !global)
                                    ? capE : 0,
                                W, ncat);
    bool const listed = global && buildItemList(W, ncat, items, words, capE);
    int maxR = 0;
    for (int gi = g0; gi < g1; ++gi) maxR = max(maxR, G[gi].mcnt / NS);
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        Item const it = listed ? itemFromList(W, items, q0 + lane)
                               : itemOf(W, ncat, q0 + lane);
        bool const active = it.gi >= 0;
        DevGroup const& g = G[active ? it.gi : g0];
        int const t = it.t;
        int const nr = active ? g.mcnt / NS : 0;
        R const rij = W.d[t];
        R const rc = R(g.rc);
        bool const valid = active && (rij < rc);
        R const dr1[3] = {W.dx[t], W.dy[t], W.dz[t]};
        R const invij = W.inv[t];
        R const pfcij = W.fc[t];
        R const pdfcrij = W.dfcr[t];
        // Shape parameters (identical for every run of the group).
        R lam[NS], zl[NS];
        int zi[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s)
        {
            DevMember const& mm = M[g.mbeg + s];
            lam[s] = R(mm.lambda);
            zl[s] = R(mm.zetaLambda);
            zi[s] = mm.zetaInt;
        }
        for (int rb = 0; rb < maxR; rb += NRC)
        {
            R aG[NRC][NS], aP1[NRC][NS], aPx[NRC][NS], aPy[NRC][NS],
              aPz[NRC][NS];
#pragma unroll
            for (int r = 0; r < NRC; ++r)
#pragma unroll
                for (int s = 0; s < NS; ++s)
                {
                    aG[r][s] = R(0);
                    aP1[r][s] = R(0);
                    aPx[r][s] = R(0);
                    aPy[r][s] = R(0);
                    aPz[r][s] = R(0);
                }
            R eta2[NRC], etaN[NRC];
            R const* Er[NRC];
#pragma unroll
            for (int r = 0; r < NRC; ++r)
            {
                int const rr = min(rb + r, max(nr - 1, 0));
                DevMember const& mm = M[g.mbeg + rr * NS];
                eta2[r] = R(2) * R(mm.eta);
                etaN[r] = -R(mm.eta);
                Er[r] = W.E + (long)mm.expIdx * capE;
            }
            // FP64: r_jk's cosine cutoff from power series in r_jk^2 (see
            // cosSincSeries, DevGroup::cosSeries).
            bool const series = (sizeof(R) == 8) && (CT == 1) && NARROW
                              && g.cosSeries;
            R const a2 = R(g.a2);
            if (valid && rb < nr)
            {
                R const cr0 = invij * invij;  // 1 / r_ij^2
                int const wb = it.pb >> 5;
                int const we = (it.pe + 31) >> 5;
                // One loop over the lane's partners (not one per mask
                // word): the warp's trip count is the largest partner count
                // of its lanes, not the sum of per-word maxima.
                if constexpr (PIPE)
                {
                // Software pipeline over the lane's partners: the pair part
                // of partner n + 1 (loads, r_jk cutoff series, the runs'
                // exponentials) is computed in the same block as the member
                // updates of partner n, so their independent chains
                // overlap.  The last trip computes a zero-weight copy.
                struct PairPart
                {
                    R dr3[3], cost, X1, X3, pr1, pr3, pfc;
                    R vexp[NRC];
                };
                auto pairPart = [&](int k, R wt) {
                    PairPart o;
                    R const dr2[3] = {W.dx[k], W.dy[k], W.dz[k]};
#pragma unroll
                    for (int c = 0; c < 3; ++c) o.dr3[c] = dr2[c] - dr1[c];
                    R const invik = W.inv[k];
                    R const pfcik = W.fc[k] * wt;
                    R const rinvijik = invij * invik;
                    o.cost = (dr1[0] * dr2[0] + dr1[1] * dr2[1]
                              + dr1[2] * dr2[2]) * rinvijik;
                    R r2 = R(0);
                    if (NARROW)
                    {
                        r2 = o.dr3[0] * o.dr3[0] + o.dr3[1] * o.dr3[1]
                           + o.dr3[2] * o.dr3[2];
                        R pfcjk, qjk;
                        if (series)
                        {
                            double c, sc;
                            cosSincSeries((double)(a2 * r2), c, sc);
                            pfcjk = R(0.5) * R(c) + R(0.5);
                            qjk = R(-0.5) * a2 * R(sc);
                        }
                        else
                        {
                            R const invjk = r2 > R(0) ? mrsqrt(r2) : R(0);
                            R pdfcjk;
                            cutoffFdf<R, CT>(P, g, r2 * invjk, pfcjk,
                                             pdfcjk);
                            qjk = pdfcjk * invjk;
                        }
                        o.pfc = pfcij * pfcik * pfcjk;
                        o.pr1 = pfcik * pfcjk * pdfcrij;
                        o.pr3 = pfcij * pfcik * qjk;
                    }
                    else
                    {
                        o.pfc = pfcij * pfcik;
                        o.pr1 = pfcik * pdfcrij;
                        o.pr3 = R(0);
                    }
                    o.X1 = o.pfc * (rinvijik - o.cost * cr0);
                    o.X3 = o.pfc * rinvijik;
#pragma unroll
                    for (int r = 0; r < NRC; ++r)
                    {
                        R v = Er[r][t] * Er[r][k];
                        if (NARROW) v *= mexp(etaN[r] * r2);
                        o.vexp[r] = v;
                    }
                    return o;
                };
                auto members = [&](PairPart const& o) {
                    R Y1[NRC], Y3[NRC];
#pragma unroll
                    for (int r = 0; r < NRC; ++r)
                    {
                        R const e2p = eta2[r] * o.pfc;
                        Y1[r] = o.pr1 - e2p;
                        Y3[r] = NARROW ? e2p - o.pr3 : R(0);
                    }
#pragma unroll
                    for (int s = 0; s < NS; ++s)
                    {
                        R const pl = R(1) + lam[s] * o.cost;
                        R const A = (pl <= R(0) || zi[s] < 1) ? R(0)
                                  : powInt16(pl, zi[s] - 1);
                        R const B = A * pl * o.pfc;
                        R const Z1 = zl[s] * o.X1;
                        R const Z3 = zl[s] * o.X3;
#pragma unroll
                        for (int r = 0; r < NRC; ++r)
                        {
                            R const wgt = o.vexp[r] * A;
                            aG[r][s] += o.vexp[r] * B;
                            aP1[r][s] += wgt * (Z1 + pl * Y1[r]);
                            R const p3 = wgt * (Z3 + pl * Y3[r]);
                            aPx[r][s] += p3 * o.dr3[0];
                            aPy[r][s] += p3 * o.dr3[1];
                            aPz[r][s] += p3 * o.dr3[2];
                        }
                    }
                };
                int w = wb - 1;
                unsigned m = 0u;
                auto next = [&]() -> int {
                    for (;;)
                    {
                        while (m == 0u && ++w < we)
                            m = rangeMask(NARROW ? W.bits[t * words + w]
                                                 : kFull,
                                          w, it.pb, it.pe);
                        if (m == 0u) return -1;
                        int const k = (w << 5) + __ffs(m) - 1;
                        m &= m - 1;
                        if (!NARROW && (k == t || !(W.d[k] < rc))) continue;
                        return k;
                    }
                };
                int k = next();
                if (k >= 0)
                {
                    PairPart cur = pairPart(k, R(1));
                    for (;;)
                    {
                        int const kn = next();
                        bool const more = kn >= 0;
                        PairPart const nxt = pairPart(more ? kn : k,
                                                      more ? R(1) : R(0));
                        members(cur);
                        if (!more) break;
                        cur = nxt;
                        k = kn;
                    }
                }
                }
                else
                {
                int w = wb - 1;
                unsigned m = 0u;
                for (;;)
                {
                    while (m == 0u && ++w < we)
                        m = rangeMask(NARROW ? W.bits[t * words + w] : kFull,
                                      w, it.pb, it.pe);
                    if (m == 0u) break;
                    {
                        int const k = (w << 5) + __ffs(m) - 1;
                        m &= m - 1;
                        if (!NARROW)
                        {
                            if (k == t || !(W.d[k] < rc)) continue;
                        }
                        R const dr2[3] = {W.dx[k], W.dy[k], W.dz[k]};
                        R const dr3[3] = {dr2[0] - dr1[0], dr2[1] - dr1[1],
                                          dr2[2] - dr1[2]};
                        R const invik = W.inv[k];
                        R const pfcik = W.fc[k];
                        R const rinvijik = invij * invik;
                        R const costijk = (dr1[0] * dr2[0] + dr1[1] * dr2[1]
                                           + dr1[2] * dr2[2]) * rinvijik;
                        R r2 = R(0), pfc, pr1, pr3 = R(0);
                        if (NARROW)
                        {
                            r2 = dr3[0] * dr3[0] + dr3[1] * dr3[1]
                               + dr3[2] * dr3[2];
                            // f_c(r_jk) and f_c'(r_jk) / r_jk
                            R pfcjk, qjk;
                            if (series)
                            {
                                double c, sc;
                                cosSincSeries((double)(a2 * r2), c, sc);
                                pfcjk = R(0.5) * R(c) + R(0.5);
                                qjk = R(-0.5) * a2 * R(sc);
                            }
                            else
                            {
                                R const invjk = mrsqrt(r2);
                                R pdfcjk;
                                cutoffFdf<R, CT>(P, g, r2 * invjk, pfcjk,
                                                 pdfcjk);
                                qjk = pdfcjk * invjk;
                            }
                            pfc = pfcij * pfcik * pfcjk;
                            pr1 = pfcik * pfcjk * pdfcrij;
                            pr3 = pfcij * pfcik * qjk;
                        }
                        else
                        {
                            pfc = pfcij * pfcik;
                            pr1 = pfcik * pdfcrij;
                        }
                        R const X1 = pfc * (rinvijik - costijk * cr0);
                        R const X3 = pfc * rinvijik;
                        R A[NS], B[NS], Z1[NS], Z3[NS], pl[NS];
#pragma unroll
                        for (int s = 0; s < NS; ++s)
                        {
                            pl[s] = R(1) + lam[s] * costijk;
                            constexpr bool kFixedPow = (NS == 8)
                                                    || (sizeof(R) == 4);
                            A[s] = (pl[s] <= R(0)) ? R(0)
                                   : (kFixedPow && g.powBits <= 4
                                      && zi[s] >= 1)
                                     ? powInt16(pl[s], zi[s] - 1)
                                     : powInt(pl[s], zi[s] - 1);
                            B[s] = A[s] * pl[s] * pfc;
                            Z1[s] = zl[s] * X1;
                            Z3[s] = zl[s] * X3;
                        }
#pragma unroll
                        for (int r = 0; r < NRC; ++r)
                        {
                            R vexp = Er[r][t] * Er[r][k];
                            if (NARROW) vexp *= mexp(etaN[r] * r2);
                            R const e2p = eta2[r] * pfc;
                            R const Y1 = pr1 - e2p;
                            R const Y3 = NARROW ? e2p - pr3 : R(0);
#pragma unroll
                            for (int s = 0; s < NS; ++s)
                            {
                                R const wgt = vexp * A[s];
                                aG[r][s] += vexp * B[s];
                                aP1[r][s] += wgt * (Z1[s] + pl[s] * Y1);
                                R const p3 = wgt * (Z3[s] + pl[s] * Y3);
                                aPx[r][s] += p3 * dr3[0];
                                aPy[r][s] += p3 * dr3[1];
                                aPz[r][s] += p3 * dr3[2];
                            }
                        }
                    }
                }
                }
            }
#pragma unroll
            for (int r = 0; r < NRC; ++r)
#pragma unroll
                for (int s = 0; s < NS; ++s)
                {
                    bool const has = active && (rb + r < nr);
                    DevMember const& mm =
                        M[g.mbeg + (has ? (rb + r) * NS + s : 0)];
                    R const fn = R(mm.factorNorm);
                    R const P1 = fn * aP1[r][s];
                    R const sx = P1 * dr1[0];
                    R const sy = P1 * dr1[1];
                    R const sz = P1 * dr1[2];
                    if (derivatives && has)
                    {
                        long const sl = mm.slot[it.et];
                        out[(sl * 3 + 0) * cnt + t] = -(sx + fn * aPx[r][s]);
                        out[(sl * 3 + 1) * cnt + t] = -(sy + fn * aPy[r][s]);
                        out[(sl * 3 + 2) * cnt + t] = -(sz + fn * aPz[r][s]);
                    }
                    flushBySF(W, it.key, has ? (int)mm.sf : -1,
                              R(0.5) * aG[r][s]);
                }
        }
    }
}

// N2P2B_SF_PATHS=31 forces the kernel with every path (A/B measurements).
inline int L_pathsOverride()
{
    static int const v = [] {
        char const* e = std::getenv("N2P2B_SF_PATHS");
        return e ? std::atoi(e) : 0;
    }();
    return v;
}

// Code paths compiled into a kernel instantiation (a kernel holding only the
// paths a potential uses is smaller and misses the instruction cache less).
constexpr int kPathRadial = 1, kPathFastNarrow = 2, kPathFastWide = 4,
              kPathGenNarrow = 8, kPathGenWide = 16, kPathCompRad = 32,
              kPathCompNarrow = 64, kPathCompWide = 128, kPathAll = 255;

// FP32 with up to 12 members per register chunk: at most 168 registers, so
// that three CTAs (12 warps) fit per SM.
template <typename R, int CT, int NS, int NRC, int PATHS, bool PIPE>
__global__ void __launch_bounds__(kThreads,
                                  (sizeof(R) == 4 && NS * NRC <= 12) ? 3 : 1)
sfKernel(__grid_constant__ SFParams const P, SFLaunch const L)
{
    extern __shared__ double smem0[];
    // Block-shared copy of the group and member tables when they fit
    // (dynamically indexed reads from global memory measured ~25% slower
    // overall); larger tables are read from global memory through L1.
    int const ng = P.numGroups;
    int const nm = P.numMembers;
    // Only the all-paths instantiation may read the tables from global
    // memory; the others see shared-memory pointers (LDS in the hot loops).
    bool const stage = (PATHS != kPathAll) || P.stageTables;
    std::size_t const staged = stage ? tableBytes(ng, nm) : 0;
    DevGroup const* sG = P.dGroups;
    DevMember const* sM = P.dMembers;
    if (stage)
    {
        DevGroup* tg = reinterpret_cast<DevGroup*>(smem0);
        DevMember* tm = reinterpret_cast<DevMember*>(tg + ng);
        int const* src = reinterpret_cast<int const*>(P.dGroups);
        int* dst = reinterpret_cast<int*>(tg);
        int const words = (int)(ng * sizeof(DevGroup) / sizeof(int));
        for (int k = threadIdx.x; k < words; k += kThreads) dst[k] = src[k];
        src = reinterpret_cast<int const*>(P.dMembers);
        dst = reinterpret_cast<int*>(tm);
        int const wm = (int)(nm * sizeof(DevMember) / sizeof(int));
        for (int k = threadIdx.x; k < wm; k += kThreads) dst[k] = src[k];
        sG = tg;
        sM = tm;
    }
    __syncthreads();
    char* smem = reinterpret_cast<char*>(smem0) + staged;
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;

    int const lane = threadIdx.x & 31;
    int const warp = threadIdx.x >> 5;
    int const cap = L.cap;
    int const words = (cap + 31) >> 5;
    int const maxSF = P.maxSF;
    R* wbase = reinterpret_cast<R*>(smem + (long)warp * L.warpBytes);
    WarpMem<R> W;
    W.dx = wbase;
    W.dy = W.dx + cap;
    W.dz = W.dy + cap;
    W.d = W.dz + cap;
    W.inv = W.d + cap;
    W.fc = W.inv + cap;
    W.dfcr = W.fc + cap;
    W.E = W.dfcr + cap;
    W.wpG = W.E + (long)P.maxExp * cap;
    {
        char* after = reinterpret_cast<char*>(W.wpG + maxSF);
        long const off = (after - reinterpret_cast<char*>(wbase) + 15) / 16
                       * 16;
        W.bits = reinterpret_cast<unsigned*>(
            reinterpret_cast<char*>(wbase) + off);
        long const off2 = (off + 4L * cap * words + 15) / 16 * 16;
        W.cats = reinterpret_cast<Cat*>(reinterpret_cast<char*>(wbase) + off2);
        char* const il = reinterpret_cast<char*>(W.cats)
                       + itemListOffset(cap, P.numElements);
        W.itemList = reinterpret_cast<unsigned*>(il);
        W.itemHist = reinterpret_cast<int*>(il + 4L * kItemsPerCap * cap);
    }
    W.sortCats = L.sortCats;
    R* const outG = static_cast<R*>(L.G);
    R* const outNbr = static_cast<R*>(L.dGdr);

    int const numElements = P.numElements;
    int const gw = blockIdx.x * kWarps + warp;
    int const nw = gridDim.x * kWarps;
    for (int i = gw; i < L.n; i += nw)
    {
        int const ec = L.elem[i];
        long const beg = L.nbrOff[i];
        int const cnt = L.nbrOff[i + 1] - (int)beg;
        if (cnt > cap)
        {
            if (lane == 0)
            {
                atomicOr(&L.status[ST_FLAGS], FLAG_SF_CAPACITY);
                atomicCAS(&L.status[ST_BAD_ATOM], -1, i);
            }
            continue;
        }
        int eb[kMaxElem + 1];
        eb[0] = 0;
        for (int e = 0; e < numElements; ++e)
            eb[e + 1] = eb[e] + L.nbrCountElem[(long)i * numElements + e];
        for (int e = numElements + 1; e <= kMaxElem; ++e) eb[e] = eb[numElements];
        for (int t = lane; t < cnt; t += 32)
        {
            double const dd = L.dd[beg + t];
            W.dx[t] = R(L.dx[beg + t]);
            W.dy[t] = R(L.dy[beg + t]);
            W.dz[t] = R(L.dz[beg + t]);
            W.d[t] = R(dd);
            W.inv[t] = R(1.0 / dd);
        }
        for (int k = lane; k < maxSF; k += 32) W.wpG[k] = R(0);
        __syncwarp();
        R* out = outNbr + beg * (long)P.maxSlots * 3;
        double fcRc = -1.0;
        double bitsRc = -1.0;
        int const gb = P.groupBeg[ec], ge = P.groupBeg[ec + 1];
        int g0 = gb;
        while (g0 < ge)
        {
            DevGroup const& h = sG[g0];
            int g1 = g0 + 1;
            bool const compactSeg = h.type >= 20;
            bool fast = (h.type != 2) && !compactSeg && (h.shapes == NS);
            while (g1 < ge && sG[g1].type == h.type && sG[g1].rc == h.rc
                   && g1 - g0 < segCap(h.type))
            {
                fast = fast && (sG[g1].shapes == NS);
                ++g1;
            }
            if (!compactSeg && h.rc != fcRc)
            {
                for (int t = lane; t < cnt; t += 32)
                {
                    R fc, dfc;
                    cutoffFdf<R, CT>(P, h, W.d[t], fc, dfc);
                    W.fc[t] = fc;
                    W.dfcr[t] = dfc * W.inv[t];
                }
                fcRc = h.rc;
            }
            if ((h.type == 3 || h.type == 13 || h.type == 21
                 || h.type == 24) && h.rc != bitsRc)
            {
                // Narrow-angular validity: k != t, r_ik < rc, r_jk^2 < rc^2.
                R const rc = R(h.rc), rc2 = R(h.rc2);
                for (int t = lane; t < cnt; t += 32)
                {
                    R const x = W.dx[t], y = W.dy[t], z = W.dz[t];
                    for (int w = 0; w < words; ++w)
                    {
                        unsigned m = 0u;
                        int const kb = w << 5;
                        int const ke = min(cnt, kb + 32);
                        for (int k = kb; k < ke; ++k)
                        {
                            R const a = W.dx[k] - x;
                            R const b = W.dy[k] - y;
                            R const c = W.dz[k] - z;
                            bool const ok = (k != t) && (W.d[k] < rc)
                                          && (a * a + b * b + c * c < rc2);
                            m |= (ok ? 1u : 0u) << (k - kb);
                        }
                        W.bits[t * words + w] = m;
                    }
                }
                __syncwarp();
                if (W.sortCats & 2)
                {
                    unsigned short* const order = ownerOrder(W);
                    int* const hist = reinterpret_cast<int*>(
                        order + (numElements * cap + 1) / 2 * 2);
                    for (int e2 = 0; e2 < numElements; ++e2)
                        for (int et = 0; et < numElements; ++et)
                            buildOwnerOrder(W, words, eb[et], eb[et + 1],
                                            eb[e2], eb[e2 + 1],
                                            order + e2 * cap, hist);
                }
                bitsRc = h.rc;
            }
            if (h.type != 2 && h.type != 12 && !compactSeg)
            {
                // Gaussian factors E(r) = exp(-eta (r - rs)^2) per distinct
                // (eta, rs) of the element (computed once per atom).
                for (int gi = g0; gi < g1; ++gi)
                {
                    DevGroup const& g = sG[gi];
                    for (int l = 0; l < g.mcnt; ++l)
                    {
                        DevMember const& mm = sM[g.mbeg + l];
                        if (!mm.fillExp) continue;
                        R* E = W.E + (long)mm.expIdx * cap;
                        R const eta = R(mm.eta), rs = R(mm.rs);
                        for (int t = lane; t < cnt; t += 32)
                        {
                            R const rr = W.d[t] - rs;
                            E[t] = mexp(-eta * rr * rr);
                        }
                    }
                }
            }
            __syncwarp();
            if (h.type == 2 || h.type == 12)
            {
                if (PATHS & kPathRadial)
                    radialSegment<R, kGenericChunk>(P, sG, sM, g0, g1, eb,
                                                    cnt, W, out,
                                                    L.derivatives);
                else if (lane == 0)
                    atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            }
            else if (h.type == 20 || h.type == 23)
            {
                if (PATHS & kPathCompRad)
                    compactRadialSegment<R, kGenericChunk>(
                        P, sG, sM, g0, g1, eb, cnt, W, out, L.derivatives);
                else if (lane == 0)
                    atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            }
            else if (h.type == 21 || h.type == 24)
            {
                if (PATHS & kPathCompNarrow)
                    compactAngularSegment<R, kCompactChunk, true>(
                        P, sG, sM, g0, g1, eb, cnt, words, W, out,
                        L.derivatives);
                else if (lane == 0)
                    atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            }
            else if (h.type == 22 || h.type == 25)
            {
                if (PATHS & kPathCompWide)
                    compactAngularSegment<R, kCompactChunk, false>(
                        P, sG, sM, g0, g1, eb, cnt, words, W, out,
                        L.derivatives);
                else if (lane == 0)
                    atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            }
            else if (fast && h.type == 3)
            {
                if (PATHS & kPathFastNarrow)
                    angularFast<R, CT, NS, NRC, true, PIPE>(P, sG, sM, g0, g1, eb,
                                                      cnt, words, cap, W, out,
                                                      L.derivatives);
                else if (lane == 0)
                    atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            }
            else if (fast)
            {
                if (PATHS & kPathFastWide)
                    angularFast<R, CT, NS, NRC, false, PIPE>(P, sG, sM, g0, g1, eb,
                                                       cnt, words, cap, W,
                                                       out, L.derivatives);
                else if (lane == 0)
                    atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            }
            else if (h.type == 3 || h.type == 13)
            {
                if (PATHS & kPathGenNarrow)
                    angularGeneric<R, CT, kGenericChunk, true>(
                        P, sG, sM, g0, g1, eb, cnt, words, cap, W, out,
                        L.derivatives);
                else if (lane == 0)
                    atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            }
            else
            {
                if (PATHS & kPathGenWide)
                    angularGeneric<R, CT, kGenericChunk, false>(
                        P, sG, sM, g0, g1, eb, cnt, words, cap, W, out,
                        L.derivatives);
                else if (lane == 0)
                    atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            }
            __syncwarp();
            g0 = g1;
        }
        __syncwarp();
        int const nsf = P.numSF[ec];
        SFScale const* sc = L.scale + (long)ec * maxSF;
        for (int s = lane; s < nsf; s += 32)
        {
            SFScale const q = sc[s];
            outG[(long)i * maxSF + s] =
                R(q.smin + q.b * (q.q * (double)W.wpG[s] - q.shift));
        }
        __syncwarp();
    }
}

// Paths a potential needs for shape count NS: the kernel's own segment
// rule (consecutive groups of equal (type, rc), at most segCap(type); fast
// only if every group of the segment has NS shapes).
inline int pathsNeeded(SFParams const& P, int NS)
{
    int paths = 0;
    for (int e = 0; e < P.numElements; ++e)
    {
        int g0 = P.groupBeg[e];
        int const ge = P.groupBeg[e + 1];
        while (g0 < ge)
        {
            DevGroup const& h = P.groups[g0];
            int g1 = g0 + 1;
            bool fast = (h.type != 2) && (h.type < 20) && (h.shapes == NS);
            while (g1 < ge && P.groups[g1].type == h.type
                   && P.groups[g1].rc == h.rc && g1 - g0 < segCap(h.type))
            {
                fast = fast && (P.groups[g1].shapes == NS);
                ++g1;
            }
            if (h.type == 2 || h.type == 12) paths |= kPathRadial;
            else if (h.type == 20 || h.type == 23) paths |= kPathCompRad;
            else if (h.type == 21 || h.type == 24) paths |= kPathCompNarrow;
            else if (h.type == 22 || h.type == 25) paths |= kPathCompWide;
            else if (fast) paths |= (h.type == 3) ? kPathFastNarrow
                                                  : kPathFastWide;
            else paths |= (h.type == 3 || h.type == 13) ? kPathGenNarrow
                                                        : kPathGenWide;
            g0 = g1;
        }
    }
    return paths;
}

// Launch and occupancy helpers for one cutoff type; variant = (NS, NRC).
// Potentials of radial + product-form narrow angular groups (the usual
// layout) get the kernel without the other paths.
constexpr int kPathsCommon = kPathRadial | kPathFastNarrow;

inline bool useCommonPaths(SFParams const& P, int NS)
{
    int const need = pathsNeeded(P, NS);
    return (need & ~kPathsCommon) == 0 && P.stageTables
        && L_pathsOverride() != kPathAll;
}

template <typename R, int CT, int NS, int NRC, bool PIPE = false>
void launchVariant(SFParams const& P, SFLaunch const& L, std::size_t shm,
                   cudaStream_t s)
{
    if (useCommonPaths(P, NS))
    {
        auto k = sfKernel<R, CT, NS, NRC, kPathsCommon, PIPE>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)shm);
        k<<<L.grid, kThreads, shm, s>>>(P, L);
        return;
    }
    auto k = sfKernel<R, CT, NS, NRC, kPathAll, PIPE>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)shm);
    k<<<L.grid, kThreads, shm, s>>>(P, L);
}

template <typename R, int CT, int NS, int NRC, bool PIPE = false>
int blocksVariant(SFParams const& P, std::size_t shm)
{
    auto k = useCommonPaths(P, NS) ? sfKernel<R, CT, NS, NRC, kPathsCommon, PIPE>
                                   : sfKernel<R, CT, NS, NRC, kPathAll, PIPE>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)shm);
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, kThreads,
                                                      shm) != cudaSuccess
        || blocks < 1)
        blocks = 1;
    return blocks;
}

} // namespace sfk
} // namespace n2p2b

#include "sf_staged.cuh"

namespace n2p2b
{
namespace sfk
{

// Variants: 0 = (NS 4, NRC 3), 1 = (4, 1), 2 = (8, 1), 3 = (8, 2); 4 and
// 5 = (4, 3) and (8, 1) with the partner loop software-pipelined
// (angularFast PIPE); 6 and 7 = the staged-triplet kernel for 4 and 8
// shapes (sf_staged.cuh).
template <typename R, int CT>
void launchForCT(SFParams const& P, SFLaunch const& L, std::size_t shm,
                 cudaStream_t s, int variant)
{
    switch (variant)
    {
    case 6: launchStaged<R, CT, 4>(P, L, shm, s); break;
    case 7: launchStaged<R, CT, 8>(P, L, shm, s); break;
    case 1: launchVariant<R, CT, 4, 1>(P, L, shm, s); break;
    case 2: launchVariant<R, CT, 8, 1>(P, L, shm, s); break;
    case 3: launchVariant<R, CT, 8, 2>(P, L, shm, s); break;
    case 4: launchVariant<R, CT, 4, 3, true>(P, L, shm, s); break;
    case 5: launchVariant<R, CT, 8, 1, true>(P, L, shm, s); break;
    default: launchVariant<R, CT, 4, 3>(P, L, shm, s); break;
    }
}

template <typename R, int CT>
int blocksForCT(SFParams const& P, std::size_t shm, int variant)
{
    switch (variant)
    {
    case 6: return blocksStaged<R, CT, 4>(shm);
    case 7: return blocksStaged<R, CT, 8>(shm);
    case 1: return blocksVariant<R, CT, 4, 1>(P, shm);
    case 2: return blocksVariant<R, CT, 8, 1>(P, shm);
    case 3: return blocksVariant<R, CT, 8, 2>(P, shm);
    case 4: return blocksVariant<R, CT, 4, 3, true>(P, shm);
    case 5: return blocksVariant<R, CT, 8, 1, true>(P, shm);
    default: return blocksVariant<R, CT, 4, 3>(P, shm);
    }
}

} // namespace sfk
} // namespace n2p2b
