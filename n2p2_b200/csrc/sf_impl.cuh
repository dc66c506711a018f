// Symmetry functions and their derivatives, FP64 (plain form) -- kernel
// templates, instantiated per cutoff type by kernels_sf_ct*.cu.
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
//   * the self derivative sum_k p1(j,k) dr_ij and the value 1/2 sum_k term(j,k)
//     (each unordered pair is seen by both owners; 0.5 scales exactly),
//     folded into per-warp sums keyed by symmetry function.
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
// per eta run and one power per shape remain; each member costs 9 FP64
// operations.  Other groups take the general path, which keeps the
// reference's expression form.
//
// dG/dr layout per atom i (n neighbors, S = maxSlots):
//   dGdr[nbrOff[i]*S*3 + (slot*3 + c)*n + t]
// consecutive neighbors t are consecutive in memory: owner lanes store, and
// the force kernel loads, coalesced.
#pragma once

#include "device_common.cuh"
#include "kernels.h"

namespace n2p2b
{
namespace sfk
{

constexpr int kWarps = 4;                 // warps (atoms) per CTA

// Bytes of the block-shared group + member tables (16-byte padded).
__host__ __device__ inline std::size_t tableBytes(int ng, int nm)
{
    return ((ng * sizeof(DevGroup) + nm * sizeof(DevMember) + 15) / 16) * 16;
}
constexpr int kThreads = 32 * kWarps;
// Members per register chunk of the general paths; small so that their
// register demand stays below the product-form path's.
constexpr int kGenericChunk = 6;
constexpr unsigned kFull = 0xffffffffu;

// CutoffFunction::fdf specialized on the (global) cutoff type; CT = -1
// dispatches at run time.
template <int CT>
__device__ __forceinline__ void cutoffFdf(SFParams const& P, DevGroup const& g,
                                          double r, double& fc, double& dfc);

template <int CT>
__device__ __forceinline__ void cutoffFdfT(SFParams const& P, DevGroup const& g,
                                           double r, double& fc, double& dfc)
{
    if (r >= g.rc)
    {
        fc = 0.0;
        dfc = 0.0;
        return;
    }
    if (CT == 0)
    {
        fc = 1.0;
        dfc = 0.0;
    }
    else if (CT == 2 || CT == 3)   // CT_TANHU, CT_TANH
    {
        double const temp = tanh(1.0 - r * g.rcinv);
        double const temp2 = temp * temp;
        double const pre = (CT == 3) ? P.TANH_PRE : 1.0;
        fc = pre * temp * temp2;
        dfc = 3.0 * pre * temp2 * (temp2 - 1.0) * g.rcinv;
    }
    else
    {
        if (r < g.rci)
        {
            fc = 1.0;
            dfc = 0.0;
            return;
        }
        double const x = (r - g.rci) * g.iw;
        if (CT == 1)               // CT_COS: d/dr cos uses sin(pi x) >= 0
        {
            double s, c;
            sincospi(x, &s, &c);
            fc = 0.5 * (c + 1.0);
            dfc = -0.5 * g.iw * P.PI * s;
        }
        else
        {
            double fx, dfx;
            if (CT == 4)           // CT_EXP
            {
                double const temp = 1.0 / (x * x - 1.0);
                double const temp2 = exp(temp);
                fx = P.E * temp2;
                dfx = -2.0 * P.E * x * temp * temp * temp2;
            }
            else if (CT == 5)      // CT_POLY1
            {
                fx = (2.0 * x - 3.0) * x * x + 1.0;
                dfx = x * (6.0 * x - 6.0);
            }
            else if (CT == 6)      // CT_POLY2
            {
                double const x2 = x * x;
                fx = ((15.0 - 6.0 * x) * x - 10.0) * x * x2 + 1.0;
                dfx = x2 * ((60.0 - 30.0 * x) * x - 30.0);
            }
            else if (CT == 7)      // CT_POLY3
            {
                double const x2 = x * x;
                fx = (x * (x * (20.0 * x - 70.0) + 84.0) - 35.0) * x2 * x2
                     + 1.0;
                dfx = x2 * x * (x * (x * (140.0 * x - 420.0) + 420.0) - 140.0);
            }
            else                   // CT_POLY4
            {
                double x4 = x * x;
                x4 *= x4;
                fx = (x * (x * ((315.0 - 70.0 * x) * x - 540.0) + 420.0)
                      - 126.0) * x * x4 + 1.0;
                dfx = x4 * (x * (x * ((2520.0 - 630.0 * x) * x - 3780.0)
                                 + 2520.0) - 630.0);
            }
            fc = fx;
            dfc = dfx * g.iw;
        }
    }
}

template <int CT>
__device__ __forceinline__ void cutoffFdf(SFParams const& P, DevGroup const& g,
                                          double r, double& fc, double& dfc)
{
    if (CT >= 0)
    {
        cutoffFdfT<(CT >= 0 ? CT : 0)>(P, g, r, fc, dfc);
        return;
    }
    switch (P.cutoffType)
    {
    case 0: cutoffFdfT<0>(P, g, r, fc, dfc); break;
    case 1: cutoffFdfT<1>(P, g, r, fc, dfc); break;
    case 2: cutoffFdfT<2>(P, g, r, fc, dfc); break;
    case 3: cutoffFdfT<3>(P, g, r, fc, dfc); break;
    case 4: cutoffFdfT<4>(P, g, r, fc, dfc); break;
    case 5: cutoffFdfT<5>(P, g, r, fc, dfc); break;
    case 6: cutoffFdfT<6>(P, g, r, fc, dfc); break;
    case 7: cutoffFdfT<7>(P, g, r, fc, dfc); break;
    default: cutoffFdfT<8>(P, g, r, fc, dfc); break;
    }
}

// pow_int (libnnp/utility.cpp:292-317): exponentiation by squaring.
__device__ __forceinline__ double powInt(double x, int n)
{
    unsigned m;
    if (n < 0)
    {
        x = 1.0 / x;
        m = (unsigned)(-n);
    }
    else m = (unsigned)n;
    double result = 1.0;
    do
    {
        if (m & 1u) result *= x;
        m >>= 1;
        x *= x;
    }
    while (m);
    return result;
}

__device__ __forceinline__ double wsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Per-warp shared-memory views.
struct WarpMem
{
    double*   dx;
    double*   dy;
    double*   dz;
    double*   d;
    double*   inv;    // 1 / d
    double*   fc;
    double*   dfcr;   // dfc / d
    double*   E;      // [expIdx][cap]
    unsigned* bits;   // [owner][words]
    double*   wpG;    // [maxSF]
    double*   wpS;    // [maxSF][3]
    struct Cat*  cats;  // work-item categories of the current segment
    int          sortCats;  // order angular categories by partner count
};

// A category is a group together with one owner element: its items are the
// owners t in [ob, ob + on) and each iterates partners in [pb, pe).
struct Cat
{
    int gi, et, ob, on, pb, pe;
};
// Segments hold at most kMaxSegGroups groups (longer runs of equal (type, rc)
// are split), so the category table never overflows.
constexpr int kMaxSegGroups = 16;
constexpr int kMaxCats = 2 * kMaxSegGroups;

// Adds each lane's (G, self) contribution for symmetry function `sf` (-1 =
// nothing) into the warp sums.  `key` identifies the lane's work-item
// category; lanes of one category occupy contiguous lanes (items are
// enumerated category by category).  One segmented butterfly reduces every
// run at once in a fixed lane order; the runs' first lanes then add their
// totals one after another (two runs may share sf).
__device__ __forceinline__ void flushBySF(WarpMem const& W, int key, int sf,
                                          double g, double sx, double sy,
                                          double sz)
{
    int const lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        double const a = __shfl_down_sync(kFull, g, off);
        double const b = __shfl_down_sync(kFull, sx, off);
        double const c = __shfl_down_sync(kFull, sy, off);
        double const e = __shfl_down_sync(kFull, sz, off);
        int const ko = __shfl_down_sync(kFull, key, off);
        if (lane + off < 32 && ko == key)
        {
            g += a;
            sx += b;
            sy += c;
            sz += e;
        }
    }
    int const prev = __shfl_up_sync(kFull, key, 1);
    bool const head = (lane == 0) || (prev != key);
    unsigned heads = __ballot_sync(kFull, head && sf >= 0);
    while (heads)
    {
        if (lane == __ffs(heads) - 1)
        {
            W.wpG[sf] += g;
            W.wpS[3 * sf + 0] += sx;
            W.wpS[3 * sf + 1] += sy;
            W.wpS[3 * sf + 2] += sz;
        }
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
__device__ __forceinline__ int buildCats(DevGroup const* G, int g0, int g1,
                                         int const eb[kMaxElem + 1],
                                         bool byPartners, WarpMem const& W,
                                         int& ncat)
{
    int const lane = threadIdx.x & 31;
    int n = 0, total = 0;
    if (lane == 0)
    {
        for (int gi = g0; gi < g1; ++gi)
        {
            DevGroup const& g = G[gi];
            int const sides = (g.type == 2 || g.e1 == g.e2) ? 1 : 2;
            for (int sd = 0; sd < sides; ++sd)
            {
                int const et = (sd == 0) ? g.e1 : g.e2;
                int const pe2 = (g.type == 2) ? g.e1
                              : ((sd == 0) ? g.e2 : g.e1);
                Cat c;
                c.gi = gi;
                c.et = et;
                c.ob = eb[et];
                c.on = eb[et + 1] - eb[et];
                c.pb = eb[pe2];
                c.pe = eb[pe2 + 1];
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

__device__ __forceinline__ Item itemOf(WarpMem const& W, int ncat, int q)
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
            it.t = cc.ob + q;
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
__device__ __forceinline__ unsigned rangeMask(unsigned m, int w, int pb, int pe)
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

template <int MC>
__device__ void radialSegment(DevGroup const* G, DevMember const* M, int g0,
                              int g1, int const eb[kMaxElem + 1], int cnt,
                              WarpMem const& W, double* __restrict__ out,
                              int derivatives)
{
    int const lane = threadIdx.x & 31;
    int ncat = 0;
    int const items = buildCats(G, g0, g1, eb, false, W, ncat);
    int maxM = 0;
    for (int gi = g0; gi < g1; ++gi) maxM = max(maxM, G[gi].mcnt);
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        Item const it = itemOf(W, ncat, q0 + lane);
        bool const active = it.gi >= 0;
        DevGroup const& g = G[active ? it.gi : g0];
        int const t = it.t;
        double const r = W.d[t];
        bool const valid = active && (r < g.rc);
        double const pfc = W.fc[t], pdfcr = W.dfcr[t], inv = W.inv[t];
        double const d1[3] = {W.dx[t], W.dy[t], W.dz[t]};
        for (int mb = 0; mb < maxM; mb += MC)
        {
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                bool const has = active && (mb + l < g.mcnt);
                DevMember const& m = M[g.mbeg + (has ? mb + l : 0)];
                double gs = 0.0, p1 = 0.0;
                if (has && valid)
                {
                    // SymGrpExpRad.cpp:210-211 with (f_c' - 2 eta (r - rs) f_c)/r
                    // written as f_c'/r - 2 eta (r - rs) f_c / r.
                    double const rr = r - m.rs;
                    double const pexp = exp(-m.eta * rr * rr);
                    gs = pexp * pfc;
                    p1 = m.factorNorm * (pdfcr - 2.0 * m.eta * rr * pfc * inv)
                       * pexp;
                }
                double const sx = p1 * d1[0], sy = p1 * d1[1], sz = p1 * d1[2];
                if (derivatives && has)
                {
                    long const s = m.slot[it.et];
                    out[(s * 3 + 0) * cnt + t] = -sx;
                    out[(s * 3 + 1) * cnt + t] = -sy;
                    out[(s * 3 + 2) * cnt + t] = -sz;
                }
                flushBySF(W, it.key, has ? (int)m.sf : -1, gs, sx, sy, sz);
            }
        }
    }
}

// General angular path: the reference's per-member expression form.
template <int CT, int MC, bool NARROW>
__device__ void angularGeneric(SFParams const& P, DevGroup const* G,
                               DevMember const* M, int g0, int g1,
                               int const eb[kMaxElem + 1], int cnt, int words,
                               int capE, WarpMem const& W,
                               double* __restrict__ out, int derivatives)
{
    int const lane = threadIdx.x & 31;
    int ncat = 0;
    int const items = buildCats(G, g0, g1, eb, W.sortCats != 0, W, ncat);
    int maxM = 0;
    for (int gi = g0; gi < g1; ++gi) maxM = max(maxM, G[gi].mcnt);
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        Item const it = itemOf(W, ncat, q0 + lane);
        bool const active = it.gi >= 0;
        DevGroup const& g = G[active ? it.gi : g0];
        int const t = it.t;
        double const rij = W.d[t];
        bool const valid = active && (rij < g.rc);
        double const dr1[3] = {W.dx[t], W.dy[t], W.dz[t]};
        double const invij = W.inv[t];
        double const pfcij = W.fc[t];
        double const pdfcrij = W.dfcr[t];
        double const rc = g.rc;
        for (int mb = 0; mb < maxM; mb += MC)
        {
            int const mc = active ? min(MC, g.mcnt - mb) : 0;
            double aG[MC], aP1[MC], aPx[MC], aPy[MC], aPz[MC];
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                aG[l] = 0.0;
                aP1[l] = 0.0;
                aPx[l] = 0.0;
                aPy[l] = 0.0;
                aPz[l] = 0.0;
            }
            if (valid && mc > 0)
            {
                double const cr0 = invij * invij;  // 1 / r_ij^2
                int const wb = it.pb >> 5;
                int const we = (it.pe + 31) >> 5;
                for (int w = wb; w < we; ++w)
                {
                    unsigned m = NARROW ? W.bits[t * words + w] : kFull;
                    m = rangeMask(m, w, it.pb, it.pe);
                    while (m)
                    {
                        int const k = (w << 5) + __ffs(m) - 1;
                        m &= m - 1;
                        if (!NARROW)
                        {
                            if (k == t || !(W.d[k] < rc)) continue;
                        }
                        double const dr2[3] = {W.dx[k], W.dy[k], W.dz[k]};
                        double const dr3[3] = {dr2[0] - dr1[0], dr2[1] - dr1[1],
                                               dr2[2] - dr1[2]};
                        double const invik = W.inv[k];
                        double const pfcik = W.fc[k];
                        double const rinvijik = invij * invik;
                        double const costijk = (dr1[0] * dr2[0] + dr1[1] * dr2[1]
                                                + dr1[2] * dr2[2]) * rinvijik;
                        double const cr = costijk * cr0;
                        double rjk = 0.0, invjk = 0.0, pfcjk = 1.0,
                               pdfcjk = 0.0;
                        if (NARROW)
                        {
                            double const r2 = dr3[0] * dr3[0] + dr3[1] * dr3[1]
                                            + dr3[2] * dr3[2];
                            invjk = rsqrt(r2);
                            rjk = r2 * invjk;
                            cutoffFdf<CT>(P, g, rjk, pfcjk, pdfcjk);
                        }
                        double pfc, pr1, pr3 = 0.0;
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
                        double vexp = 0.0;
#pragma unroll
                        for (int l = 0; l < MC; ++l)
                        {
                            if (l >= mc) break;
                            DevMember const& mm = M[g.mbeg + mb + l];
                            if (mm.calcExp || l == 0)
                            {
                                double const* E = W.E + (long)mm.expIdx * capE;
                                vexp = E[t] * E[k];
                                if (NARROW)
                                {
                                    double const rjks = rjk - mm.rs;
                                    vexp *= exp(-mm.eta * rjks * rjks);
                                }
                            }
                            double const plambda = 1.0 + mm.lambda * costijk;
                            double fg = vexp;
                            if (plambda <= 0.0) fg = 0.0;
                            else if (mm.useIntPow)
                                fg *= powInt(plambda, mm.zetaInt - 1);
                            else
                                fg *= pow(plambda, mm.zeta - 1.0);
                            aG[l] += fg * plambda * pfc;
                            fg *= mm.factorNorm;
                            double const pfczl = pfc * mm.zetaLambda;
                            double const p2etapl = plambda * mm.factorDeriv;
                            double p1, p3;
                            if (mm.rsPositive)
                            {
                                double const rijs = rij - mm.rs;
                                p1 = fg * (pfczl * (rinvijik - cr
                                                    - p2etapl * rijs * invij)
                                           + pr1 * plambda);
                                if (NARROW)
                                {
                                    double const rjks = rjk - mm.rs;
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
                double const sx = aP1[l] * dr1[0];
                double const sy = aP1[l] * dr1[1];
                double const sz = aP1[l] * dr1[2];
                if (derivatives && has)
                {
                    long const s = mm.slot[it.et];
                    out[(s * 3 + 0) * cnt + t] = -(sx + aPx[l]);
                    out[(s * 3 + 1) * cnt + t] = -(sy + aPy[l]);
                    out[(s * 3 + 2) * cnt + t] = -(sz + aPz[l]);
                }
                flushBySF(W, it.key, has ? (int)mm.sf : -1, 0.5 * aG[l], sx,
                          sy, sz);
            }
        }
    }
}

// Product-form angular path (see the header comment): NS shapes per eta
// run, NRC runs per register chunk.
template <int CT, int NS, int NRC, bool NARROW>
__device__ void angularFast(SFParams const& P, DevGroup const* G,
                            DevMember const* M, int g0, int g1,
                            int const eb[kMaxElem + 1], int cnt, int words,
                            int capE, WarpMem const& W,
                            double* __restrict__ out, int derivatives)
{
    int const lane = threadIdx.x & 31;
    int ncat = 0;
    int const items = buildCats(G, g0, g1, eb, W.sortCats != 0, W, ncat);
    int maxR = 0;
    for (int gi = g0; gi < g1; ++gi) maxR = max(maxR, G[gi].mcnt / NS);
    for (int q0 = 0; q0 < items; q0 += 32)
    {
        Item const it = itemOf(W, ncat, q0 + lane);
        bool const active = it.gi >= 0;
        DevGroup const& g = G[active ? it.gi : g0];
        int const t = it.t;
        int const nr = active ? g.mcnt / NS : 0;
        double const rij = W.d[t];
        bool const valid = active && (rij < g.rc);
        double const dr1[3] = {W.dx[t], W.dy[t], W.dz[t]};
        double const invij = W.inv[t];
        double const pfcij = W.fc[t];
        double const pdfcrij = W.dfcr[t];
        double const rc = g.rc;
        // Shape parameters (identical for every run of the group).
        double lam[NS], zl[NS];
        int zi[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s)
        {
            DevMember const& mm = M[g.mbeg + s];
            lam[s] = mm.lambda;
            zl[s] = mm.zetaLambda;
            zi[s] = mm.zetaInt;
        }
        for (int rb = 0; rb < maxR; rb += NRC)
        {
            double aG[NRC][NS], aP1[NRC][NS], aPx[NRC][NS], aPy[NRC][NS],
                   aPz[NRC][NS];
#pragma unroll
            for (int r = 0; r < NRC; ++r)
#pragma unroll
                for (int s = 0; s < NS; ++s)
                {
                    aG[r][s] = 0.0;
                    aP1[r][s] = 0.0;
                    aPx[r][s] = 0.0;
                    aPy[r][s] = 0.0;
                    aPz[r][s] = 0.0;
                }
            double eta2[NRC], etaN[NRC];
            double const* Er[NRC];
#pragma unroll
            for (int r = 0; r < NRC; ++r)
            {
                int const rr = min(rb + r, max(nr - 1, 0));
                DevMember const& mm = M[g.mbeg + rr * NS];
                eta2[r] = 2.0 * mm.eta;
                etaN[r] = -mm.eta;
                Er[r] = W.E + (long)mm.expIdx * capE;
            }
            if (valid && rb < nr)
            {
                double const cr0 = invij * invij;  // 1 / r_ij^2
                int const wb = it.pb >> 5;
                int const we = (it.pe + 31) >> 5;
                for (int w = wb; w < we; ++w)
                {
                    unsigned m = NARROW ? W.bits[t * words + w] : kFull;
                    m = rangeMask(m, w, it.pb, it.pe);
                    while (m)
                    {
                        int const k = (w << 5) + __ffs(m) - 1;
                        m &= m - 1;
                        if (!NARROW)
                        {
                            if (k == t || !(W.d[k] < rc)) continue;
                        }
                        double const dr2[3] = {W.dx[k], W.dy[k], W.dz[k]};
                        double const dr3[3] = {dr2[0] - dr1[0], dr2[1] - dr1[1],
                                               dr2[2] - dr1[2]};
                        double const invik = W.inv[k];
                        double const pfcik = W.fc[k];
                        double const rinvijik = invij * invik;
                        double const costijk = (dr1[0] * dr2[0] + dr1[1] * dr2[1]
                                                + dr1[2] * dr2[2]) * rinvijik;
                        double r2 = 0.0, pfc, pr1, pr3 = 0.0;
                        if (NARROW)
                        {
                            r2 = dr3[0] * dr3[0] + dr3[1] * dr3[1]
                               + dr3[2] * dr3[2];
                            double const invjk = rsqrt(r2);
                            double pfcjk, pdfcjk;
                            cutoffFdf<CT>(P, g, r2 * invjk, pfcjk, pdfcjk);
                            pfc = pfcij * pfcik * pfcjk;
                            pr1 = pfcik * pfcjk * pdfcrij;
                            pr3 = pfcij * pfcik * pdfcjk * invjk;
                        }
                        else
                        {
                            pfc = pfcij * pfcik;
                            pr1 = pfcik * pdfcrij;
                        }
                        double const X1 = pfc * (rinvijik - costijk * cr0);
                        double const X3 = pfc * rinvijik;
                        double A[NS], B[NS], Z1[NS], Z3[NS], pl[NS];
#pragma unroll
                        for (int s = 0; s < NS; ++s)
                        {
                            pl[s] = 1.0 + lam[s] * costijk;
                            A[s] = (pl[s] <= 0.0) ? 0.0 : powInt(pl[s], zi[s] - 1);
                            B[s] = A[s] * pl[s] * pfc;
                            Z1[s] = zl[s] * X1;
                            Z3[s] = zl[s] * X3;
                        }
#pragma unroll
                        for (int r = 0; r < NRC; ++r)
                        {
                            double vexp = Er[r][t] * Er[r][k];
                            if (NARROW) vexp *= exp(etaN[r] * r2);
                            double const e2p = eta2[r] * pfc;
                            double const Y1 = pr1 - e2p;
                            double const Y3 = NARROW ? e2p - pr3 : 0.0;
#pragma unroll
                            for (int s = 0; s < NS; ++s)
                            {
                                double const wgt = vexp * A[s];
                                aG[r][s] += vexp * B[s];
                                aP1[r][s] += wgt * (Z1[s] + pl[s] * Y1);
                                double const p3 = wgt * (Z3[s] + pl[s] * Y3);
                                aPx[r][s] += p3 * dr3[0];
                                aPy[r][s] += p3 * dr3[1];
                                aPz[r][s] += p3 * dr3[2];
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
                    double const fn = mm.factorNorm;
                    double const P1 = fn * aP1[r][s];
                    double const sx = P1 * dr1[0];
                    double const sy = P1 * dr1[1];
                    double const sz = P1 * dr1[2];
                    if (derivatives && has)
                    {
                        long const sl = mm.slot[it.et];
                        out[(sl * 3 + 0) * cnt + t] = -(sx + fn * aPx[r][s]);
                        out[(sl * 3 + 1) * cnt + t] = -(sy + fn * aPy[r][s]);
                        out[(sl * 3 + 2) * cnt + t] = -(sz + fn * aPz[r][s]);
                    }
                    flushBySF(W, it.key, has ? (int)mm.sf : -1, 0.5 * aG[r][s],
                              sx, sy,
                              sz);
                }
        }
    }
}

template <int CT, int NS, int NRC>
__global__ void __launch_bounds__(kThreads)
sfFp64Kernel(__grid_constant__ SFParams const P, SFLaunch const L)
{
    extern __shared__ double smem0[];
    // Block-shared copy of the group and member tables (dynamically indexed
    // reads from the parameter bank measured ~25% slower overall).
    int const ng = P.groupBeg[P.numElements];
    int nm = 0;
    if (ng > 0) nm = P.groups[ng - 1].mbeg + P.groups[ng - 1].mcnt;
    DevGroup* tg = reinterpret_cast<DevGroup*>(smem0);
    DevMember* tm = reinterpret_cast<DevMember*>(tg + ng);
    {
        int const* src = reinterpret_cast<int const*>(P.groups);
        int* dst = reinterpret_cast<int*>(tg);
        int const words = (int)(ng * sizeof(DevGroup) / sizeof(int));
        for (int k = threadIdx.x; k < words; k += kThreads) dst[k] = src[k];
        src = reinterpret_cast<int const*>(P.members);
        dst = reinterpret_cast<int*>(tm);
        int const wm = (int)(nm * sizeof(DevMember) / sizeof(int));
        for (int k = threadIdx.x; k < wm; k += kThreads) dst[k] = src[k];
    }
    __syncthreads();
    double* smem = reinterpret_cast<double*>(
        reinterpret_cast<char*>(smem0) + tableBytes(ng, nm));
    DevGroup const* sG = tg;
    DevMember const* sM = tm;
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;

    int const lane = threadIdx.x & 31;
    int const warp = threadIdx.x >> 5;
    int const cap = L.cap;
    int const words = (cap + 31) >> 5;
    int const maxSF = P.maxSF;
    double* wbase = smem + (long)warp * L.warpDoubles;
    WarpMem W;
    W.dx = wbase;
    W.dy = W.dx + cap;
    W.dz = W.dy + cap;
    W.d = W.dz + cap;
    W.inv = W.d + cap;
    W.fc = W.inv + cap;
    W.dfcr = W.fc + cap;
    W.E = W.dfcr + cap;
    W.wpG = W.E + (long)P.maxExp * cap;
    W.wpS = W.wpG + maxSF;
    W.bits = reinterpret_cast<unsigned*>(W.wpS + 3 * maxSF);
    W.cats = reinterpret_cast<Cat*>(W.bits + cap * words);
    W.sortCats = L.sortCats;

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
            W.dx[t] = L.dx[beg + t];
            W.dy[t] = L.dy[beg + t];
            W.dz[t] = L.dz[beg + t];
            W.d[t] = dd;
            W.inv[t] = 1.0 / dd;
        }
        for (int k = lane; k < 4 * maxSF; k += 32) W.wpG[k] = 0.0;
        __syncwarp();
        double* out = L.dGdr + beg * (long)P.maxSlots * 3;
        double fcRc = -1.0;
        double bitsRc = -1.0;
        int const gb = P.groupBeg[ec], ge = P.groupBeg[ec + 1];
        int g0 = gb;
        while (g0 < ge)
        {
            DevGroup const& h = sG[g0];
            int g1 = g0 + 1;
            bool fast = (h.type != 2) && (h.shapes == NS);
            while (g1 < ge && sG[g1].type == h.type && sG[g1].rc == h.rc
                   && g1 - g0 < kMaxSegGroups)
            {
                fast = fast && (sG[g1].shapes == NS);
                ++g1;
            }
            if (h.rc != fcRc)
            {
                for (int t = lane; t < cnt; t += 32)
                {
                    double fc, dfc;
                    cutoffFdf<CT>(P, h, W.d[t], fc, dfc);
                    W.fc[t] = fc;
                    W.dfcr[t] = dfc * W.inv[t];
                }
                fcRc = h.rc;
            }
            if (h.type == 3 && h.rc != bitsRc)
            {
                // Narrow-angular validity: k != t, r_ik < rc, r_jk^2 < rc^2.
                double const rc = h.rc, rc2 = h.rc2;
                for (int t = lane; t < cnt; t += 32)
                {
                    double const x = W.dx[t], y = W.dy[t], z = W.dz[t];
                    for (int w = 0; w < words; ++w)
                    {
                        unsigned m = 0u;
                        int const kb = w << 5;
                        int const ke = min(cnt, kb + 32);
                        for (int k = kb; k < ke; ++k)
                        {
                            double const a = W.dx[k] - x;
                            double const b = W.dy[k] - y;
                            double const c = W.dz[k] - z;
                            bool const ok = (k != t) && (W.d[k] < rc)
                                          && (a * a + b * b + c * c < rc2);
                            m |= (ok ? 1u : 0u) << (k - kb);
                        }
                        W.bits[t * words + w] = m;
                    }
                }
                bitsRc = h.rc;
            }
            if (h.type != 2)
            {
                // Gaussian factors E(r) = exp(-eta (r - rs)^2) per distinct
                // (eta, rs) run of the segment's members.
                for (int gi = g0; gi < g1; ++gi)
                {
                    DevGroup const& g = sG[gi];
                    for (int l = 0; l < g.mcnt; ++l)
                    {
                        DevMember const& mm = sM[g.mbeg + l];
                        if (!mm.calcExp) continue;
                        double* E = W.E + (long)mm.expIdx * cap;
                        for (int t = lane; t < cnt; t += 32)
                        {
                            double const rr = W.d[t] - mm.rs;
                            E[t] = exp(-mm.eta * rr * rr);
                        }
                    }
                }
            }
            __syncwarp();
            if (h.type == 2)
                radialSegment<kGenericChunk>(sG, sM, g0, g1, eb, cnt, W, out,
                                             L.derivatives);
            else if (fast && h.type == 3)
                angularFast<CT, NS, NRC, true>(P, sG, sM, g0, g1, eb, cnt,
                                               words, cap, W, out,
                                               L.derivatives);
            else if (fast)
                angularFast<CT, NS, NRC, false>(P, sG, sM, g0, g1, eb, cnt,
                                                words, cap, W, out,
                                                L.derivatives);
            else if (h.type == 3)
                angularGeneric<CT, kGenericChunk, true>(
                    P, sG, sM, g0, g1, eb, cnt, words, cap, W, out,
                    L.derivatives);
            else
                angularGeneric<CT, kGenericChunk, false>(
                    P, sG, sM, g0, g1, eb, cnt, words, cap, W, out,
                    L.derivatives);
            __syncwarp();
            g0 = g1;
        }
        __syncwarp();
        int const nsf = P.numSF[ec];
        SFScale const* sc = L.scale + (long)ec * maxSF;
        for (int s = lane; s < nsf; s += 32)
        {
            SFScale const q = sc[s];
            L.G[(long)i * maxSF + s] = q.smin + q.b * (q.q * W.wpG[s] - q.shift);
            if (L.derivatives)
            {
                double* o = L.dGdrSelf + ((long)i * maxSF + s) * 3;
                o[0] = W.wpS[3 * s + 0];
                o[1] = W.wpS[3 * s + 1];
                o[2] = W.wpS[3 * s + 2];
            }
        }
        __syncwarp();
    }
}

// Launch and occupancy helpers for one cutoff type; variant = (NS, NRC).
template <int CT, int NS, int NRC>
void launchVariant(SFParams const& P, SFLaunch const& L, std::size_t shm,
                   cudaStream_t s)
{
    cudaFuncSetAttribute(sfFp64Kernel<CT, NS, NRC>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    sfFp64Kernel<CT, NS, NRC><<<L.grid, kThreads, shm, s>>>(P, L);
}

template <int CT, int NS, int NRC>
int blocksVariant(std::size_t shm)
{
    cudaFuncSetAttribute(sfFp64Kernel<CT, NS, NRC>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &blocks, sfFp64Kernel<CT, NS, NRC>, kThreads, shm) != cudaSuccess
        || blocks < 1)
        blocks = 1;
    return blocks;
}

// Variants: 0 = (NS 4, NRC 3), 1 = (4, 1), 2 = (8, 1), 3 = (8, 2).
template <int CT>
void launchForCT(SFParams const& P, SFLaunch const& L, std::size_t shm,
                 cudaStream_t s, int variant)
{
    switch (variant)
    {
    case 1: launchVariant<CT, 4, 1>(P, L, shm, s); break;
    case 2: launchVariant<CT, 8, 1>(P, L, shm, s); break;
    case 3: launchVariant<CT, 8, 2>(P, L, shm, s); break;
    default: launchVariant<CT, 4, 3>(P, L, shm, s); break;
    }
}

template <int CT>
int blocksForCT(std::size_t shm, int variant)
{
    switch (variant)
    {
    case 1: return blocksVariant<CT, 4, 1>(shm);
    case 2: return blocksVariant<CT, 8, 1>(shm);
    case 3: return blocksVariant<CT, 8, 2>(shm);
    default: return blocksVariant<CT, 4, 3>(shm);
    }
}

} // namespace sfk
} // namespace n2p2b
