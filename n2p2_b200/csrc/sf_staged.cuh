// Staged-triplet symmetry-function kernel for product-form narrow angular
// groups (SymGrpExpAngn, libnnp/SymGrpExpAngn.cpp:156-403) and radial groups
// (SymGrpExpRad, libnnp/SymGrpExpRad.cpp:144-239).  Included by
// sf_impl.cuh, whose helpers it uses.
//
// Decomposition: one CTA (4 warps) per central atom i, persistent grid.  The
// atom's neighbors are staged once per CTA (1/r, f_c, f_c'/r, the exp
// tables) and shared by the four warps, which split the atom's work items
// (group, owner neighbor j) round robin.  A warp runs each batch of its
// items in two phases:
//
//   phase 1 (lanes over triplets): for every valid partner k of the batch's
//     owners, the member-independent part of the triplet (j, k) is computed
//     once and stored as a record in the warp's shared memory:
//       v_a   = E_a(r_ij) E_a(r_ik) exp(-eta_a r_jk^2)      per eta run a
//       beta  = A plambda pfc                                per shape s
//       alpha'= A (zl X1 + plambda pr1) - gamma              per shape s
//       gamma = A (zl X3 - plambda pr3)                      per shape s
//       r_ik  (3 components)
//     with the quantities of the product form (sf_impl.cuh: A = plambda^
//     (zeta - 1), X1, X3, pfc, pr1, pr3);
//   phase 2 (lanes over (member, partner slice)): lane (m, s) of member
//     m = (run a, shape s) sums over every S-th record of the owner
//       G  += v beta
//       Q  += v (alpha' - 4 eta beta)        (= p1 - p3)
//       V  += v (gamma + 2 eta beta) r_ik    (= p3 r_ik)
//     so that the owner's slot is -(fn (Q r_ij + V)); the S partial sums of
//     a member are added in slice order (fixed), then written once.
//
// Per (triplet, member) this leaves five FP64 accumulations and their
// operands' loads; the member-independent work (r_jk's cutoff, the runs'
// exponentials, the shape powers) is done once per ordered triplet, and no
// lane holds more than five accumulators, so the kernel runs at four CTAs
// (16 warps) per SM instead of the per-owner kernel's 8 warps.  All sums
// are formed in a fixed order: results are deterministic run to run.
#pragma once

#include <algorithm>

namespace n2p2b
{
namespace sfk
{

// Work items (owners) per batch (a batch also ends when its records fill
// the buffer).
constexpr int kStagedItems = 32;
constexpr int kStagedThreads = kThreads;   // 4 warps, one atom
constexpr int kStagedWarps = kWarps;
// eta runs per group the records hold (groups have at most this many).
constexpr int kStagedRuns = 4;
// Dynamic shared memory per CTA the record capacity is sized for: four CTAs
// per SM, less the exponential's table (static, 512 bytes)
// (N2P2B_SF_STAGED_KB overrides it, in KB, for measurements).
constexpr long kStagedTargetBytes = 56L * 1024 - 512;
inline long stagedTargetBytes()
{
    static long const v = [] {
        char const* e = std::getenv("N2P2B_SF_STAGED_KB");
        return e ? std::atol(e) * 1024L : kStagedTargetBytes;
    }();
    return v;
}

__host__ __device__ inline long align16(long b) { return (b + 15) / 16 * 16; }

// Record of one ordered triplet (values of the compute type):
//   [0, 3)                 r_ik
//   [3 + 3 s, 6 + 3 s)     beta, alpha', gamma of shape s
//   [3 + 3 NS + a]         v of eta run a
// The stride is odd and, with 4 shapes (two partner slices read one load
// instruction), puts the two slices' shape fields on disjoint banks.
__host__ __device__ constexpr int stagedStride(int ns)
{
    return ns == 4 ? 21 : 3 + 3 * ns + kStagedRuns;
}

// Per-category constants of phase 1, shared by the warp's lanes; 16-byte
// aligned fields, read in FP64 as pairs (lambda, zeta lambda), (eta, eta),
// (a^2 / 4, -a^2 / 2) and quadruples of ints.
template <typename R, int NS>
struct alignas(16) StagedCat
{
    static_assert(NS % 4 == 0, "shapes in quadruples");
    R   lz[2 * NS];          // lambda, zeta lambda of shape s at 2 s, 2 s + 1
    R   eta[kStagedRuns];
    int zi[NS];
    int eoff[kStagedRuns];   // offset of the run's exp table in W.E
    R   a2q, qf;             // a^2 / 4 and -a^2 / 2, a = pi / rc (the
                             // FP64 cosine cutoff's series)
    DevGroup grp;            // the group (its cutoff parameters)
};

// Per-warp region: G sums, categories, batch list and tables, category
// constants, records, and the lockstep path's partner lists (one list of
// up to cap partners per owner of a group of 32 / ns owners), owner order
// (cap entries) and its 32 sort buckets.
template <typename R>
__host__ __device__ inline long stagedWarpBytes(int maxSF, int ns, int rb,
                                                int cap)
{
    long b = align16((long)sizeof(R) * maxSF);
    b += kCatsBytes;
    b += align16(4L * rb + 4L * (2 * kStagedItems + 1));
    b += align16(ns == 4 ? (long)sizeof(StagedCat<R, 4>)
                         : (long)sizeof(StagedCat<R, 8>));
    b += align16((long)sizeof(R) * stagedStride(ns) * rb);
    b += align16(2L * (32 / ns) * cap + 2L * cap);
    b += 4L * 32;
    return b;
}

// Atom-shared region: staged neighbors and the narrow validity bits.
template <typename R>
__host__ __device__ inline long stagedAtomBytes(int maxExp, int cap)
{
    long const words = (cap + 31) / 32;
    return align16((long)sizeof(R) * (7L + maxExp) * cap)
         + align16(4L * cap * words);
}

// tables: the group and member tables are staged in shared memory (else
// read from global memory through L1).
template <typename R>
__host__ __device__ inline long stagedSharedBytes(SFParams const& P, int cap,
                                                  int ns, int rb, bool tables)
{
    return (tables ? (long)stagedTableBytes(P) : 0L)
         + stagedAtomBytes<R>(P.maxExp, cap)
         + kStagedWarps * stagedWarpBytes<R>(P.maxSF, ns, rb, cap);
}

// The staged kernel serves potentials whose groups are radial or
// product-form narrow angular with ns shapes, at most kStagedRuns eta runs
// and at most 32 members (one lane each).
inline bool stagedEligible(SFParams const& P, int ns)
{
    if ((pathsNeeded(P, ns) & ~(kPathRadial | kPathFastNarrow)) != 0)
        return false;
    for (int g = 0; g < P.groupBeg[P.numElements]; ++g)
    {
        DevGroup const& h = P.groups[g];
        if (h.type == 3
            && (h.shapes != ns || h.mcnt > 32 || h.mcnt % ns
                || h.mcnt / ns > kStagedRuns))
            return false;
    }
    return true;
}

// Record capacity: the largest multiple of 16 in [32, 96] whose CTA fits
// stagedTargetBytes() (32 when none does).
template <typename R>
inline int stagedRecordCap(SFParams const& P, int cap, int ns, bool tables)
{
    for (int rb = 96; rb > 32; rb -= 16)
        if (stagedSharedBytes<R>(P, cap, ns, rb, tables)
            <= stagedTargetBytes())
            return rb;
    return 32;
}

// The tables are staged in shared memory when the CTA fits
// stagedTargetBytes() with the smallest record capacity; larger tables (the
// 92-SF potential's) are read from global memory, which keeps four CTAs
// per SM.
template <typename R>
inline bool stagedTablesShared(SFParams const& P, int cap, int ns)
{
    return P.stageTables
        && stagedSharedBytes<R>(P, cap, ns, 32, true) <= stagedTargetBytes();
}

// 2^(j / 64), j = 0 .. 63, rounded to nearest: the table of the exponential
// below, staged into shared memory by the kernels that use it.
static __constant__ double kExp2Table[64] = {
    0x1.0000000000000p+0, 0x1.02c9a3e778061p+0, 0x1.059b0d3158574p+0,
    0x1.0874518759bc8p+0, 0x1.0b5586cf9890fp+0, 0x1.0e3ec32d3d1a2p+0,
    0x1.11301d0125b51p+0, 0x1.1429aaea92de0p+0, 0x1.172b83c7d517bp+0,
    0x1.1a35beb6fcb75p+0, 0x1.1d4873168b9aap+0, 0x1.2063b88628cd6p+0,
    0x1.2387a6e756238p+0, 0x1.26b4565e27cddp+0, 0x1.29e9df51fdee1p+0,
    0x1.2d285a6e4030bp+0, 0x1.306fe0a31b715p+0, 0x1.33c08b26416ffp+0,
    0x1.371a7373aa9cbp+0, 0x1.3a7db34e59ff7p+0, 0x1.3dea64c123422p+0,
    0x1.4160a21f72e2ap+0, 0x1.44e086061892dp+0, 0x1.486a2b5c13cd0p+0,
    0x1.4bfdad5362a27p+0, 0x1.4f9b2769d2ca7p+0, 0x1.5342b569d4f82p+0,
    0x1.56f4736b527dap+0, 0x1.5ab07dd485429p+0, 0x1.5e76f15ad2148p+0,
    0x1.6247eb03a5585p+0, 0x1.6623882552225p+0, 0x1.6a09e667f3bcdp+0,
    0x1.6dfb23c651a2fp+0, 0x1.71f75e8ec5f74p+0, 0x1.75feb564267c9p+0,
    0x1.7a11473eb0187p+0, 0x1.7e2f336cf4e62p+0, 0x1.82589994cce13p+0,
    0x1.868d99b4492edp+0, 0x1.8ace5422aa0dbp+0, 0x1.8f1ae99157736p+0,
    0x1.93737b0cdc5e5p+0, 0x1.97d829fde4e50p+0, 0x1.9c49182a3f090p+0,
    0x1.a0c667b5de565p+0, 0x1.a5503b23e255dp+0, 0x1.a9e6b5579fdbfp+0,
    0x1.ae89f995ad3adp+0, 0x1.b33a2b84f15fbp+0, 0x1.b7f76f2fb5e47p+0,
    0x1.bcc1e904bc1d2p+0, 0x1.c199bdd85529cp+0, 0x1.c67f12e57d14bp+0,
    0x1.cb720dcef9069p+0, 0x1.d072d4a07897cp+0, 0x1.d5818dcfba487p+0,
    0x1.da9e603db3285p+0, 0x1.dfc97337b9b5fp+0, 0x1.e502ee78b3ff6p+0,
    0x1.ea4afa2a490dap+0, 0x1.efa1bee615a27p+0, 0x1.f50765b6e4540p+0,
    0x1.fa7c1819e90d8p+0,
};
constexpr int kExpTableSize = 64;

// exp(x) for x <= 0 in FP64 without branches, by Tang's table-driven method
// (P. T. P. Tang, ACM TOMS 15 (1989) 144-157): x = (64 m + j) ln2 / 64 + r,
// |r| <= ln2 / 128, with ln2 / 64 split into a 32-bit head (k ln2_hi exact
// for |k| < 2^21) and a tail; exp(x) = 2^m T[j] (1 + q), q = exp(r) - 1 by
// its Taylor polynomial of degree 6 (truncation below 2.7e-20), formed as
// T[j] + T[j] q so that q's rounding hardly counts.  Within 1.01 ulp of the
// exact value where the result is normal.  Arguments below -708.39
// (m < -1022) return 0 where libm returns subnormals (< 2.3e-308).  tab is
// kExp2Table in shared memory.
__device__ __forceinline__ double expNonPositive(double x,
                                                 double const* tab)
{
    constexpr double kInvL = 0x1.71547652b82fep+6;     // 64 / ln2
    constexpr double kLHi = 0x1.62e42fee00000p-7;      // ln2 / 64, head
    constexpr double kLLo = 0x1.a39ef35793c76p-39;     // ln2 / 64, tail
    constexpr double kShift = 0x1.8p52;
    double const t = fma(x, kInvL, kShift);
    int const k = __double2loint(t);
    double const kd = t - kShift;
    double r = fma(-kd, kLHi, x);
    r = fma(-kd, kLLo, r);
    double const r2 = r * r;
    double p = fma(r, InvFact<6>::value, InvFact<5>::value);
    p = fma(p, r, InvFact<4>::value);
    p = fma(p, r, InvFact<3>::value);
    p = fma(p, r, 0.5);
    double const q = fma(p, r2, r);
    double const tj = tab[k & (kExpTableSize - 1)];
    // m < -1022 gives two = +0 (the clamp to -1023 zeroes the exponent).
    int const m = max(k >> 6, -1023);
    double const two = __hiloint2double((m + 1023) << 20, 0);
    return fma(tj, q, tj) * two;
}
__device__ __forceinline__ float expNonPositive(float x, double const*)
{
    return __expf(x);
}

// pow_int (libnnp/utility.cpp:292-317) for the shape exponents zeta - 1 of
// a record's group, which are the same in every lane of the warp (a batch or
// lockstep group holds one category): zeta = 1, 2, 4, 8, 16 as straight
// multiplication chains in pow_int's order (bit-identical results), other
// exponents through the branch-free powInt16 / the loop.  FP32 keeps the
// branch-free form throughout (measured faster there: its selects are
// single instructions).
template <typename R>
__device__ __forceinline__ R powShape(R x, int n)
{
    if (sizeof(R) == 4)
        return (n >= 0 && n < 16) ? powInt16(x, n) : powInt(x, n);
    switch (n)
    {
    case 0: return R(1);
    case 1: return x;
    case 3:
    {
        R const x2 = x * x;
        return x * x2;
    }
    case 7:
    {
        R const x2 = x * x;
        R const x4 = x2 * x2;
        return (x * x2) * x4;
    }
    case 15:
    {
        R const x2 = x * x;
        R const x4 = x2 * x2;
        R const x8 = x4 * x4;
        return ((x * x2) * x4) * x8;
    }
    default:
        return (n >= 0 && n < 16) ? powInt16(x, n) : powInt(x, n);
    }
}

// The owner's staged values a record reads (loaded once per owner).
template <typename R>
struct StagedOwner
{
    R dr[3], inv, fc, dfcr;
    R E[kStagedRuns];   // E_a(r_ij) of the group's eta runs
};

template <typename R, int NS>
__device__ __forceinline__ StagedOwner<R> stagedOwner(WarpMem<R> const& W,
                                                      StagedCat<R, NS> const& C,
                                                      int nr, int t)
{
    StagedOwner<R> v;
    v.dr[0] = W.dx[t];
    v.dr[1] = W.dy[t];
    v.dr[2] = W.dz[t];
    v.inv = W.inv[t];
    v.fc = W.fc[t];
    v.dfcr = W.dfcr[t];
#pragma unroll
    for (int a = 0; a < kStagedRuns; ++a)
        v.E[a] = (a < nr) ? W.E[C.eoff[a] + t] : R(0);
    return v;
}

// Phase 1: the record of ordered triplet (owner t, partner k) of a group
// with constants C; HOIST: the owner's values come from ow (else they are
// read from the staged arrays here).
template <typename R, int CT, int NS, bool HOIST>
__device__ __forceinline__ void stagedRecord(SFParams const& P,
                                             DevGroup const& g,
                                             StagedCat<R, NS> const& C,
                                             int nr, bool series, int t,
                                             StagedOwner<R> const& ow, int k,
                                             WarpMem<R> const& W,
                                             R* __restrict__ rec)
{
    R const dr1[3] = {HOIST ? ow.dr[0] : W.dx[t], HOIST ? ow.dr[1] : W.dy[t],
                      HOIST ? ow.dr[2] : W.dz[t]};
    R const dr2[3] = {W.dx[k], W.dy[k], W.dz[k]};
    R const invij = HOIST ? ow.inv : W.inv[t];
    R const pfcij = HOIST ? ow.fc : W.fc[t];
    R const pfcik = W.fc[k];
    R const pdfcrij = HOIST ? ow.dfcr : W.dfcr[t];
    R const dr3[3] = {dr2[0] - dr1[0], dr2[1] - dr1[1], dr2[2] - dr1[2]};
    R const rinvijik = invij * W.inv[k];
    R const cost = (dr1[0] * dr2[0] + dr1[1] * dr2[1] + dr1[2] * dr2[2])
                 * rinvijik;
    R const r2 = dr3[0] * dr3[0] + dr3[1] * dr3[1] + dr3[2] * dr3[2];
    // f_c(r_jk) and f_c'(r_jk) / r_jk (FP64 cosine cutoff: half-angle power
    // series in r_jk^2, see halfAngleCosSinc).
    R pfcjk, qjk;
    if ((sizeof(R) == 8) && (CT == 1) && series)
    {
        double2 const aq = *reinterpret_cast<double2 const*>(&C.a2q);
        double ch, sh;
        halfAngleCosSinc(aq.x * (double)r2, ch, sh);
        pfcjk = R(ch * ch);
        qjk = R(aq.y * (sh * ch));
    }
    else
    {
        R const invjk = mrsqrt(r2);
        R pdfcjk;
        cutoffFdf<R, CT>(P, g, r2 * invjk, pfcjk, pdfcjk);
        qjk = pdfcjk * invjk;
    }
    // alpha' = A (zl X1 + plambda pr1) - gamma with gamma = A (zl X3 -
    // plambda pr3) is A zl (X1 - X3) + D (pr1 + pr3), D = A plambda, and
    // X1 - X3 = -pfc cos / r_ij^2.
    R const fijik = pfcij * pfcik;
    R const pfc = fijik * pfcjk;
    R const pr1 = pfcik * pfcjk * pdfcrij;
    R const pr3 = fijik * qjk;
    R const pr13 = pr1 + pr3;
    R const Xc = -(pfc * cost) * (invij * invij);
    R const X3 = pfc * rinvijik;
    rec[0] = dr2[0];
    rec[1] = dr2[1];
    rec[2] = dr2[2];
    // The category's constants: pairs and quadruples in FP64.
    int zis[NS];
#pragma unroll
    for (int q = 0; q < NS / 4; ++q)
    {
        int4 const v = reinterpret_cast<int4 const*>(C.zi)[q];
        zis[4 * q] = v.x;
        zis[4 * q + 1] = v.y;
        zis[4 * q + 2] = v.z;
        zis[4 * q + 3] = v.w;
    }
#pragma unroll
    for (int s = 0; s < NS; ++s)
    {
        R lam, zls;
        if constexpr (sizeof(R) == 8)
        {
            double2 const v = reinterpret_cast<double2 const*>(C.lz)[s];
            lam = v.x;
            zls = v.y;
        }
        else
        {
            lam = C.lz[2 * s];
            zls = C.lz[2 * s + 1];
        }
        int const zi = zis[s];
        R const pl = R(1) + lam * cost;
        R const A = (pl <= R(0)) ? R(0) : powShape(pl, zi - 1);
        R const D = A * pl;
        R const Azl = A * zls;
        rec[3 + 3 * s] = D * pfc;
        rec[4 + 3 * s] = Azl * Xc + D * pr13;
        rec[5 + 3 * s] = Azl * X3 - D * pr3;
    }
#pragma unroll
    for (int a = 0; a < kStagedRuns; ++a)
        if (a < nr)
        {
            R const* E = W.E + C.eoff[a];
            rec[3 + 3 * NS + a] = (HOIST ? ow.E[a] : E[t]) * E[k]
                                * expNonPositive(-C.eta[a] * r2, W.expTab);
        }
}

// A product-form narrow angular segment [g0, g1).  Categories (group, owner
// element) are walked in order; warp w takes owners w, w + warps, ... of
// each, in batches of owners whose partners fill at most rb records.
template <typename R, int CT, int NS>
__device__ void stagedNarrow(SFParams const& P, DevGroup const* G,
                             DevMember const* M, int g0, int g1,
                             int const eb[kMaxElem + 1], int cnt, int words,
                             int capE, WarpMem<R> const& W, int* list,
                             int* bT, int* bOff, StagedCat<R, NS>* cp,
                             R* recs, int rb, int warp, int warps,
                             R* __restrict__ out, int derivatives)
{
    constexpr int NF = stagedStride(NS);
    int const lane = threadIdx.x & 31;
    unsigned const below = (1u << lane) - 1u;
    int ncat = 0;
    buildCats(G, g0, g1, eb, false, 0, W, ncat);
    for (int c = 0; c < ncat; ++c)
    {
        Cat const cc = W.cats[c];
        DevGroup const& g = G[cc.gi];
        // Owners beyond the group's cutoff have no triplets; their slots
        // are written as zero like the others'.
        R const rc = R(g.rc);
        int const mc = g.mcnt;
        int const nr = mc / NS;
        bool const series = g.cosSeries != 0;
        if (lane == 0)
        {
            for (int s = 0; s < NS; ++s)
            {
                DevMember const& mm = M[g.mbeg + s];
                cp->lz[2 * s] = R(mm.lambda);
                cp->lz[2 * s + 1] = R(mm.zetaLambda);
                cp->zi[s] = mm.zetaInt;
            }
            for (int a = 0; a < kStagedRuns; ++a)
            {
                DevMember const& mm = M[g.mbeg + min(a, nr - 1) * NS];
                cp->eta[a] = R(mm.eta);
                cp->eoff[a] = mm.expIdx * capE;
            }
            cp->a2q = R(0.25) * R(g.a2);
            cp->qf = R(-0.5) * R(g.a2);
        }
        // Phase-2 lane: member m of slice s (S slices of the partners).
        int const S = 32 / mc;
        int const s = lane / mc;
        int const m = lane - s * mc;
        bool const p2 = s < S;
        int const a = m / NS;
        int const sh = m - a * NS;
        DevMember const& lm = M[g.mbeg + (p2 ? m : 0)];
        R const eta = R(M[g.mbeg + a * NS].eta);
        R const eta2 = R(2) * eta, eta4 = R(4) * eta;
        R const fn = R(lm.factorNorm);
        R* const outL = out + (long)lm.slot[cc.et] * 3 * cnt;
        R* const gL = W.wpG + lm.sf;
        int const offS = 3 + 3 * sh;
        int const offV = 3 + 3 * NS + a;
        __syncwarp();
        StagedCat<R, NS> const& C = *cp;

        // Sums of the open owner (carried across batches when its partners
        // span more than one).
        R aG = R(0), aQ = R(0), aX = R(0), aY = R(0), aZ = R(0);
        int o = warp;
        int wcur = -1;   // word to resume the open owner at
        while (o < cc.on)
        {
            // ---- phase 0: the batch's partner list, whole mask words ----
            int n = 0, nb = 0;
            bool open = false;
            while (o < cc.on && nb < kStagedItems)
            {
                int const t = cc.ob + o;
                int w = (wcur >= 0) ? wcur : (cc.pb >> 5);
                int const we = (W.d[t] < rc) ? (cc.pe + 31) >> 5 : w;
                if (lane == 0)
                {
                    bT[nb] = t;
                    bOff[nb] = n;
                }
                for (; w < we; ++w)
                {
                    unsigned const mk = rangeMask(W.bits[t * words + w], w,
                                                  cc.pb, cc.pe);
                    int const cw = __popc(mk);
                    if (n + cw > rb) break;
                    if ((mk >> lane) & 1u)
                        list[n + __popc(mk & below)] = (nb << 16)
                                                     | ((w << 5) + lane);
                    n += cw;
                }
                ++nb;
                if (w < we)
                {
                    wcur = w;
                    open = true;
                    break;
                }
                wcur = -1;
                o += warps;
            }
            if (lane == 0) bOff[nb] = n;
            __syncwarp();
            // ---- phase 1: one record per ordered triplet --------------
            for (int r = lane; r < n; r += 32)
            {
                int const e = list[r];
                stagedRecord<R, CT, NS, false>(P, g, C, nr, series,
                                               bT[e >> 16], StagedOwner<R>(),
                                               e & 0xffff, W,
                                               recs + (long)r * NF);
            }
            __syncwarp();
            // ---- phase 2: lanes (member, slice) over each owner ---------
            for (int b = 0; b < nb; ++b)
            {
                int const ro = bOff[b], re = bOff[b + 1];
                if (p2)
                {
                    R const* q = recs + (long)(ro + s) * NF;
#pragma unroll 2
                    for (int r = ro + s; r < re; r += S, q += S * NF)
                    {
                        R const v = q[offV];
                        R const be = q[offS];
                        aG += v * be;
                        aQ += v * (q[offS + 1] - eta4 * be);
                        R const p3 = v * (q[offS + 2] + eta2 * be);
                        aX += p3 * q[0];
                        aY += p3 * q[1];
                        aZ += p3 * q[2];
                    }
                }
                if (b < nb - 1 || !open)
                {
                    // The owner ends here: slice sums in slice order, then
                    // the member's slot and value.
                    for (int s2 = 1; s2 < S; ++s2)
                    {
                        int const src = (lane + s2 * mc) & 31;
                        aG += __shfl_sync(kFull, aG, src);
                        aQ += __shfl_sync(kFull, aQ, src);
                        aX += __shfl_sync(kFull, aX, src);
                        aY += __shfl_sync(kFull, aY, src);
                        aZ += __shfl_sync(kFull, aZ, src);
                    }
                    if (lane < mc)
                    {
                        int const t = bT[b];
                        if (derivatives)
                        {
                            outL[t] = -(fn * (aQ * W.dx[t] + aX));
                            outL[cnt + t] = -(fn * (aQ * W.dy[t] + aY));
                            outL[2 * cnt + t] = -(fn * (aQ * W.dz[t] + aZ));
                        }
                        *gL += R(0.5) * aG;
                    }
                    aG = aQ = aX = aY = aZ = R(0);
                }
            }
            __syncwarp();
        }
    }
}

// Radial groups (SymGrpExpRad, libnnp/SymGrpExpRad.cpp:144-239, and the
// element-weighted type 12) of segment [g0, g1).  Per category (group,
// neighbor element) lane (member m, sub-lane u) of warp w takes neighbors
// ob + w S + u, ob + (w + warps) S + u, ... (S = 32 / members sub-lanes),
// writes the member's slot of each and sums its G terms in that order; the
// S sums of a member are then added by a fixed tree and the member's G
// gets the total once per category.  Neighbors beyond the group's cutoff
// get zero slots.
template <typename R>
__device__ void stagedRadial(SFParams const& P, DevGroup const* G,
                             DevMember const* M, int g0, int g1,
                             int const eb[kMaxElem + 1], int cnt,
                             WarpMem<R> const& W, R* __restrict__ out,
                             int derivatives, int warp, int warps)
{
    int const lane = threadIdx.x & 31;
    for (int gi = g0; gi < g1; ++gi)
    {
        DevGroup const& g = G[gi];
        bool const weighted = g.type == 12;
        R const rc = R(g.rc);
        for (int et = 0; et < kMaxElem; ++et)
        {
            int const ob = eb[et], oe = eb[et + 1];
            if (weighted ? (oe <= ob) : (et != g.e1)) continue;
            R const z = weighted ? R(P.atomicNumber[et]) : R(1);
            for (int mb = 0; mb < g.mcnt; mb += 32)
            {
                int const mn = min(32, g.mcnt - mb);
                int const S = 32 / mn;
                int const u = lane / mn;
                int const m = mb + lane - u * mn;
                bool const act = u < S;
                DevMember const& mm = M[g.mbeg + (act ? m : mb)];
                R const eta = R(mm.eta), rs = R(mm.rs);
                R const fn = R(mm.factorNorm);
                R* const o3 = out + (long)mm.slot[et] * 3 * cnt;
                R gs = R(0);
                if (act)
                    for (int t = ob + warp * S + u; t < oe; t += warps * S)
                    {
                        R const r = W.d[t];
                        R p1 = R(0);
                        if (r < rc)
                        {
                            // SymGrpExpRad.cpp:210-211 with (f_c' - 2 eta
                            // (r - rs) f_c) / r written as f_c' / r - 2 eta
                            // (r - rs) f_c / r.
                            R const rr = r - rs;
                            R const pfc = W.fc[t];
                            R const pexp = z * expNonPositive(-eta * rr * rr,
                                                              W.expTab);
                            gs += pexp * pfc;
                            p1 = fn * (W.dfcr[t] - R(2) * eta * rr * pfc
                                                   * W.inv[t]) * pexp;
                        }
                        if (derivatives)
                        {
                            o3[t] = -(p1 * W.dx[t]);
                            o3[cnt + t] = -(p1 * W.dy[t]);
                            o3[2 * cnt + t] = -(p1 * W.dz[t]);
                        }
                    }
                for (int d = 1; d < S; d <<= 1)
                {
                    R const v = __shfl_down_sync(kFull, gs, d * mn);
                    if ((u & (2 * d - 1)) == 0 && u + d < S) gs += v;
                }
                if (u == 0) W.wpG[mm.sf] += gs;
                __syncwarp();
            }
        }
    }
}

// Eta runs per group the lockstep path keeps in registers.
constexpr int kLockRuns = 3;

// A product-form narrow angular segment [g0, g1) in lockstep: the warp runs
// groups of J = 32 / NS owners of a category at once, and lane
// (owner o = lane / NS, x = lane % NS) plays two roles per step of NS
// partners:
//   phase 1: the record of owner o's (step NS + x)-th valid partner;
//   phase 2: the members (run a, shape x), a < runs, of owner o, summed
//            over owner o's NS records of the step.
// Every (owner, member) pair lives in one lane for the whole group: no
// slice sums, one slot write per member when the group ends.  The group's
// G values are added over its owners by a fixed butterfly.  Groups of a
// category go to the warps round robin; an owner's partners come from a
// list built from its validity mask (lanes of the owner split each mask
// word).  Records of partners beyond an owner's count carry v = 0.  The
// owners of a category are taken in the order of their partner counts
// (descending; buildOwnerOrder, one warp per category for the whole CTA),
// so that a group's owners need about the same number of steps.  The
// groups of the segment's categories, heaviest first within a category, are
// dealt to the warps in snake order (0 .. w-1, w-1 .. 0, ...) continued
// across the categories, which evens out the warps' work before the CTA's
// barrier at the segment's end.
template <typename R, int CT, int NS>
__device__ void stagedNarrowLock(SFParams const& P, DevGroup const* G,
                                 DevMember const* M, int g0, int g1,
                                 int const eb[kMaxElem + 1], int cnt,
                                 int words, int capE, WarpMem<R> const& W,
                                 StagedCat<R, NS>* cp, R* recs,
                                 unsigned short* plist,
                                 unsigned short* order, int* hist,
                                 long warpStride, int warp, int warps,
                                 R* __restrict__ out, int derivatives)
{
    constexpr int NF = stagedStride(NS);
    constexpr int J = 32 / NS;
    int const lane = threadIdx.x & 31;
    int const o = lane / NS;
    int const x = lane - o * NS;
    unsigned short* const myList = plist + o * capE;
    R* const myRec = recs + lane * NF;
    int ncat = 0;
    buildCats(G, g0, g1, eb, false, 0, W, ncat);
    int dealt = 0;   // groups dealt so far in this segment
    // Categories in chunks of `warps`: warp w orders category cb + w's
    // owners into its own order array, which every warp of the CTA then
    // reads (CTA barriers around each chunk; ncat is the same in every
    // warp).
    for (int cb = 0; cb < ncat; cb += warps)
    {
    if (cb + warp < ncat)
    {
        Cat const cs = W.cats[cb + warp];
        buildOwnerOrder(W, words, cs.ob, cs.ob + cs.on, cs.pb, cs.pe, order,
                        hist);
    }
    __syncthreads();
    for (int c = cb; c < min(cb + warps, ncat); ++c)
    {
        Cat const cc = W.cats[c];
        unsigned short const* const ord = reinterpret_cast<unsigned short*>(
            reinterpret_cast<char*>(order) + (long)(c - cb - warp)
                                             * warpStride);
        int const ng = (cc.on + J - 1) / J;
        int const first = dealt;
        dealt += ng;
        // Does this warp get any of the category's groups?
        bool mine = false;
        for (int k = 0; k < ng && !mine; ++k)
        {
            int const pos = (first + k) % warps;
            int const rnd = (first + k) / warps;
            mine = ((rnd & 1) ? warps - 1 - pos : pos) == warp;
        }
        if (!mine) continue;
        DevGroup const& g = G[cc.gi];
        R const rc = R(g.rc);
        int const nr = g.mcnt / NS;
        bool const series = g.cosSeries != 0;
        // The category's constants, one field set per lane.
        if (lane < NS)
        {
            DevMember const& mm = M[g.mbeg + lane];
            cp->lz[2 * lane] = R(mm.lambda);
            cp->lz[2 * lane + 1] = R(mm.zetaLambda);
            cp->zi[lane] = mm.zetaInt;
        }
        else if (lane < NS + kStagedRuns)
        {
            int const a = lane - NS;
            DevMember const& mm = M[g.mbeg + min(a, nr - 1) * NS];
            cp->eta[a] = R(mm.eta);
            cp->eoff[a] = mm.expIdx * capE;
        }
        else if (lane == 31)
        {
            cp->grp = g;
            cp->a2q = R(0.25) * R(g.a2);
            cp->qf = R(-0.5) * R(g.a2);
        }
        __syncwarp();
        StagedCat<R, NS> const& C = *cp;
        R eta2[kLockRuns], eta4[kLockRuns];
#pragma unroll
        for (int a = 0; a < kLockRuns; ++a)
        {
            eta2[a] = R(2) * C.eta[a];
            eta4[a] = R(4) * C.eta[a];
        }
        int const wb = cc.pb >> 5;
        int const we = (cc.pe + 31) >> 5;

        for (int k = 0; k < ng; ++k)
        {
            int const pos = (first + k) % warps;
            int const rnd = (first + k) / warps;
            if (((rnd & 1) ? warps - 1 - pos : pos) != warp) continue;
            int const q0 = k * J;
            // ---- the owners' partner lists ----------------------------
            int const oi = q0 + o;
            bool const own = oi < cc.on;
            int const t = own ? (int)ord[cc.ob + oi] : cc.ob;
            // The owner's NS lanes take one mask word each per round; a
            // prefix of the words' counts over those lanes places each
            // word's partners.
            bool const act = own && W.d[t] < rc;
            // The owner's values stay in registers for the group where
            // they fit (8 shapes: 3 CTAs per SM); with 4 shapes they are
            // read per record, which keeps 4 CTAs per SM without spills.
            constexpr bool kHoist = NS == 8;
            StagedOwner<R> ow{};
            if constexpr (kHoist) ow = stagedOwner(W, C, nr, t);
            int np = 0;
            for (int w0 = wb; w0 < we; w0 += NS)
            {
                int const w = w0 + x;
                unsigned mk = (act && w < we)
                            ? rangeMask(W.bits[t * words + w], w, cc.pb,
                                        cc.pe)
                            : 0u;
                int const c = __popc(mk);
                int incl = c;
#pragma unroll
                for (int d = 1; d < NS; d <<= 1)
                {
                    int const v = __shfl_up_sync(kFull, incl, d, NS);
                    if (x >= d) incl += v;
                }
                int pos = np + incl - c;
                while (mk)
                {
                    int const bit = __ffs(mk) - 1;
                    mk &= mk - 1u;
                    myList[pos++] = (unsigned short)((w << 5) + bit);
                }
                np += __shfl_sync(kFull, incl, NS - 1, NS);
            }
            int most = np;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
                most = max(most, __shfl_xor_sync(kFull, most, off));
            __syncwarp();
            // ---- steps of NS partners per owner -----------------------
            R aG[kLockRuns], aQ[kLockRuns], aX[kLockRuns], aY[kLockRuns],
              aZ[kLockRuns];
#pragma unroll
            for (int a = 0; a < kLockRuns; ++a)
                aG[a] = aQ[a] = aX[a] = aY[a] = aZ[a] = R(0);
            for (int p0 = 0; p0 < most; p0 += NS)
            {
                int const pi = p0 + x;
                if (pi < np)
                    stagedRecord<R, CT, NS, kHoist>(P, C.grp, C, nr, series,
                                                    t, ow, myList[pi], W,
                                                    myRec);
                else
                {
#pragma unroll
                    for (int a = 0; a < kLockRuns; ++a)
                        myRec[3 + 3 * NS + a] = R(0);
                }
                __syncwarp();
#pragma unroll
                for (int j = 0; j < NS; ++j)
                {
                    R const* q = recs + (o * NS + j) * NF;
                    R const be = q[3 + 3 * x];
                    R const al = q[4 + 3 * x];
                    R const ga = q[5 + 3 * x];
                    R const rx = q[0], ry = q[1], rz = q[2];
#pragma unroll
                    for (int a = 0; a < kLockRuns; ++a)
                    {
                        R const v = q[3 + 3 * NS + a];
                        aG[a] += v * be;
                        aQ[a] += v * al;
                        R const p3 = v * (ga + eta2[a] * be);
                        aX[a] += p3 * rx;
                        aY[a] += p3 * ry;
                        aZ[a] += p3 * rz;
                    }
                }
                __syncwarp();
            }
            // ---- slots of the group's owners; G over the owners -------
#pragma unroll
            for (int a = 0; a < kLockRuns; ++a)
            {
                if (a >= nr) break;
                DevMember const& mm = M[g.mbeg + a * NS + x];
                if (own && derivatives)
                {
                    // Q = sum v (alpha' - 4 eta beta) = sum v alpha'
                    //     - 4 eta G.
                    R const fn = R(mm.factorNorm);
                    R const Q = aQ[a] - eta4[a] * aG[a];
                    R* const o3 = out + (long)mm.slot[cc.et] * 3 * cnt + t;
                    o3[0] = -(fn * (Q * W.dx[t] + aX[a]));
                    o3[cnt] = -(fn * (Q * W.dy[t] + aY[a]));
                    o3[2 * cnt] = -(fn * (Q * W.dz[t] + aZ[a]));
                }
                R gs = aG[a];
#pragma unroll
                for (int off = NS; off < 32; off <<= 1)
                    gs += __shfl_xor_sync(kFull, gs, off);
                if (o == 0) W.wpG[mm.sf] += R(0.5) * gs;
            }
            __syncwarp();
        }
    }
    __syncthreads();   // the orders are rewritten by the next chunk
    }
}

// Four CTAs (16 warps) per SM; FP64 with 8 shapes is held to three by its
// shared memory (the 92-SF potential's), and gets their registers instead
// of spilling.
template <typename R, int CT, int NS>
__global__ void __launch_bounds__(kStagedThreads,
                                  (sizeof(R) == 8 && NS == 8) ? 3 : 4)
sfStagedKernel(__grid_constant__ SFParams const P, SFLaunch const L)
{
    extern __shared__ double smem0[];
    __shared__ double expTab[sizeof(R) == 8 ? kExpTableSize : 1];
    int const ng = P.numGroups;
    int const nm = P.numMembers;
    int const tid = threadIdx.x;
    if (sizeof(R) == 8)
        for (int j = tid; j < kExpTableSize; j += kStagedThreads)
            expTab[j] = kExp2Table[j];
    // Group and member tables: staged in shared memory when they fit the
    // CTA's budget, else read from global memory through L1.
    bool const tables = L.tablesShared != 0;
    DevGroup const* sG = P.dGroups;
    DevMember const* sM = P.dMembers;
    if (tables)
    {
        DevGroup* tg = reinterpret_cast<DevGroup*>(smem0);
        DevMember* tm = reinterpret_cast<DevMember*>(tg + ng);
        int const* src = reinterpret_cast<int const*>(P.dGroups);
        int* dst = reinterpret_cast<int*>(tg);
        int const words = (int)(ng * sizeof(DevGroup) / sizeof(int));
        for (int k = tid; k < words; k += kStagedThreads) dst[k] = src[k];
        src = reinterpret_cast<int const*>(P.dMembers);
        dst = reinterpret_cast<int*>(tm);
        int const wm = (int)(nm * sizeof(DevMember) / sizeof(int));
        for (int k = tid; k < wm; k += kStagedThreads) dst[k] = src[k];
        sG = tg;
        sM = tm;
    }
    __syncthreads();
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;

    int const lane = tid & 31;
    int const warp = tid >> 5;
    int const cap = L.cap;
    int const words = (cap + 31) >> 5;
    int const maxSF = P.maxSF;
    char* const base = reinterpret_cast<char*>(smem0)
                     + (tables ? tableBytes(ng, nm) : 0);
    R* const st = reinterpret_cast<R*>(base);
    WarpMem<R> W;
    W.dx = st;
    W.dy = W.dx + cap;
    W.dz = W.dy + cap;
    W.d = W.dz + cap;
    W.inv = W.d + cap;
    W.fc = W.inv + cap;
    W.dfcr = W.fc + cap;
    W.E = W.dfcr + cap;
    W.bits = reinterpret_cast<unsigned*>(
        base + align16((long)sizeof(R) * (7L + P.maxExp) * cap));
    W.expTab = expTab;
    char* const warps0 = base + stagedAtomBytes<R>(P.maxExp, cap);
    char* const wp = warps0 + (long)warp * L.warpBytes;
    W.wpG = reinterpret_cast<R*>(wp);
    W.cats = reinterpret_cast<Cat*>(wp + align16((long)sizeof(R) * maxSF));
    W.itemList = nullptr;
    W.itemHist = nullptr;
    W.sortCats = 0;
    int const rb = L.recCap;
    int* const list = reinterpret_cast<int*>(reinterpret_cast<char*>(W.cats)
                                             + kCatsBytes);
    int* const bT = list + rb;
    int* const bOff = bT + kStagedItems;
    char* const cpp = reinterpret_cast<char*>(list)
                    + align16(4L * rb + 4L * (2 * kStagedItems + 1));
    StagedCat<R, NS>* const cp = reinterpret_cast<StagedCat<R, NS>*>(cpp);
    R* const recs = reinterpret_cast<R*>(
        cpp + align16((long)sizeof(StagedCat<R, NS>)));
    unsigned short* const plist = reinterpret_cast<unsigned short*>(
        reinterpret_cast<char*>(recs)
        + align16((long)sizeof(R) * stagedStride(NS) * rb));
    unsigned short* const order = plist + (32 / NS) * cap;
    int* const hist = reinterpret_cast<int*>(
        reinterpret_cast<char*>(plist)
        + align16(2L * (32 / NS) * cap + 2L * cap));
    // The lockstep path writes only the runs' values of padding records:
    // every record starts finite.
    for (int k = lane; k < 32 * stagedStride(NS); k += 32) recs[k] = R(0);
    __syncwarp();
    R* const outG = static_cast<R*>(L.G);
    R* const outNbr = static_cast<R*>(L.dGdr);
    int const numElements = P.numElements;

    for (int i = blockIdx.x; i < L.n; i += gridDim.x)
    {
        int const ec = L.elem[i];
        long const beg = L.nbrOff[i];
        int const cnt = L.nbrOff[i + 1] - (int)beg;
        if (cnt > cap)
        {
            if (tid == 0)
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
        for (int t = tid; t < cnt; t += kStagedThreads)
        {
            double const dd = L.dd[beg + t];
            W.dx[t] = R(L.dx[beg + t]);
            W.dy[t] = R(L.dy[beg + t]);
            W.dz[t] = R(L.dz[beg + t]);
            W.d[t] = R(dd);
            W.inv[t] = R(1.0 / dd);
        }
        for (int k = lane; k < maxSF; k += 32) W.wpG[k] = R(0);
        __syncthreads();
        R* out = outNbr + beg * (long)P.maxSlots * 3;
        double fcRc = -1.0;
        double bitsRc = -1.0;
        int const gb = P.groupBeg[ec], ge = P.groupBeg[ec + 1];
        int g0 = gb;
        while (g0 < ge)
        {
            DevGroup const& h = sG[g0];
            int g1 = g0 + 1;
            while (g1 < ge && sG[g1].type == h.type && sG[g1].rc == h.rc
                   && g1 - g0 < segCap(h.type))
                ++g1;
            if (h.rc != fcRc)
            {
                for (int t = tid; t < cnt; t += kStagedThreads)
                {
                    R fc, dfc;
                    cutoffFdf<R, CT>(P, h, W.d[t], fc, dfc);
                    W.fc[t] = fc;
                    W.dfcr[t] = dfc * W.inv[t];
                }
                fcRc = h.rc;
            }
            if (h.type == 3 && h.rc != bitsRc)
            {
                // Narrow-angular validity: k != t, r_ik < rc, r_jk^2 < rc^2.
                // Warp v takes rows t = v, v + warps, ...; lane l holds the
                // partners k = 32 w + l of four words at a time, and each
                // word is a ballot (only the words holding partners,
                // ceil(cnt / 32), are formed; no one reads the others).
                R const rc = R(h.rc), rc2 = R(h.rc2);
                int const wn = (cnt + 31) >> 5;
                for (int w0 = 0; w0 < wn; w0 += 4)
                {
                    R xk[4], yk[4], zk[4];
                    bool okk[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                    {
                        int const k = ((w0 + j) << 5) + lane;
                        int const kk = k < cnt ? k : 0;
                        okk[j] = (k < cnt) && (W.d[kk] < rc);
                        xk[j] = W.dx[kk];
                        yk[j] = W.dy[kk];
                        zk[j] = W.dz[kk];
                    }
                    for (int t = warp; t < cnt; t += kStagedWarps)
                    {
                        R const xt = W.dx[t], yt = W.dy[t], zt = W.dz[t];
                        unsigned m[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                        {
                            R const a = xk[j] - xt;
                            R const b = yk[j] - yt;
                            R const c = zk[j] - zt;
                            bool const ok = okk[j]
                                          && (((w0 + j) << 5) + lane != t)
                                          && (a * a + b * b + c * c < rc2);
                            m[j] = __ballot_sync(kFull, ok);
                        }
                        unsigned const mine = lane == 0 ? m[0]
                                            : lane == 1 ? m[1]
                                            : lane == 2 ? m[2] : m[3];
                        if (lane < min(4, wn - w0))
                            W.bits[t * words + w0 + lane] = mine;
                    }
                }
                bitsRc = h.rc;
            }
            if (h.type == 3)
            {
                // E(r) = exp(-eta (r - rs)^2) per distinct (eta, rs) of the
                // element.
                for (int gi = g0; gi < g1; ++gi)
                {
                    DevGroup const& g = sG[gi];
                    for (int l = 0; l < g.mcnt; ++l)
                    {
                        DevMember const& mm = sM[g.mbeg + l];
                        if (!mm.fillExp) continue;
                        R* E = W.E + (long)mm.expIdx * cap;
                        R const eta = R(mm.eta), rs = R(mm.rs);
                        for (int t = tid; t < cnt; t += kStagedThreads)
                        {
                            R const rr = W.d[t] - rs;
                            E[t] = mexp(-eta * rr * rr);
                        }
                    }
                }
            }
            __syncthreads();
            if (h.type == 2 || h.type == 12)
                stagedRadial<R>(P, sG, sM, g0, g1, eb, cnt, W, out,
                                L.derivatives, warp, kStagedWarps);
            else if (h.type == 3 && h.shapes == NS)
            {
                int runs = 0;
                for (int gi = g0; gi < g1; ++gi)
                    runs = max(runs, sG[gi].mcnt / NS);
                if (L.lockstep && runs <= kLockRuns)
                    stagedNarrowLock<R, CT, NS>(P, sG, sM, g0, g1, eb, cnt,
                                                words, cap, W, cp, recs,
                                                plist, order, hist,
                                                L.warpBytes, warp,
                                                kStagedWarps, out,
                                                L.derivatives);
                else
                    stagedNarrow<R, CT, NS>(P, sG, sM, g0, g1, eb, cnt, words,
                                            cap, W, list, bT, bOff, cp, recs,
                                            rb, warp, kStagedWarps, out,
                                            L.derivatives);
            }
            else if (tid == 0)
                atomicOr(&L.status[ST_FLAGS], FLAG_SF_PATH);
            __syncthreads();
            g0 = g1;
        }
        // G: the warps' sums in warp order, then the scaling transform.
        int const nsf = P.numSF[ec];
        SFScale const* sc = L.scale + (long)ec * maxSF;
        for (int s = tid; s < nsf; s += kStagedThreads)
        {
            R v = R(0);
            for (int w = 0; w < kStagedWarps; ++w)
                v += reinterpret_cast<R const*>(warps0 + (long)w
                                                * L.warpBytes)[s];
            SFScale const q = sc[s];
            outG[(long)i * maxSF + s] =
                R(q.smin + q.b * (q.q * (double)v - q.shift));
        }
        __syncthreads();
    }
}

template <typename R, int CT, int NS>
void launchStaged(SFParams const& P, SFLaunch const& L, std::size_t shm,
                  cudaStream_t s)
{
    auto k = sfStagedKernel<R, CT, NS>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)shm);
    k<<<L.grid, kStagedThreads, shm, s>>>(P, L);
}

template <typename R, int CT, int NS>
int blocksStaged(std::size_t shm)
{
    auto k = sfStagedKernel<R, CT, NS>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)shm);
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k,
                                                      kStagedThreads, shm)
            != cudaSuccess
        || blocks < 1)
        blocks = 1;
    return blocks;
}

} // namespace sfk
} // namespace n2p2b
