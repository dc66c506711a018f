// Symmetry functions and their derivatives, FP64 (plain form).
//
// Semantics: Element::calculateSymmetryFunctionGroups driving
//   SymGrpExpRad::calculate   (libnnp/SymGrpExpRad.cpp:144-239)   type 2
//   SymGrpExpAngn::calculate  (libnnp/SymGrpExpAngn.cpp:156-403)  type 3
//   SymGrpExpAngw::calculate  (libnnp/SymGrpExpAngw.cpp:156-376)  type 9
// with CutoffFunction::fdf (libnnp/CutoffFunction.cpp:128-213) and
// CoreFunction (libnnp/CoreFunction.h:171-320).  The per-pair and per-member
// expressions keep the reference's association so results agree to rounding.
//
// Decomposition (B200): one CTA per central atom i at a time (persistent
// grid).  The atom's neighbor displacements, distances and cutoff values are
// staged in shared memory, grouped by neighbor element (the neighbor list is
// stored element-grouped).  Each thread OWNS one neighbor j and loops over the
// partners k of the group's other element:
//   * dG/dr slot of j:  -(sum_k p1(j,k)) dr_ij - sum_k p3(j,k) (dr_ik - dr_ij)
//     accumulated in registers, written once (single writer, no atomics);
//   * self derivative:  sum_j (sum_k p1(j,k)) dr_ij   (warp-shuffle reduction)
//   * G:                1/2 sum_j sum_k term(j,k)     (each unordered pair is
//     seen by both of its owners; 0.5 scales exactly).
// For the ordered pair (j as first) p1 is the reference's p1 and for j as
// second the reference's p2 -- the same expression with roles swapped -- so
// every stored value is the reference's value up to summation order.
// Block-level sums are formed per warp and added in warp order: the result is
// deterministic run to run.
//
// dG/dr layout per atom i (n neighbors, S = maxSlots):
//   dGdr[nbrOff[i]*S*3 + (slot*3 + c)*n + t]
// so that consecutive neighbors t are consecutive in memory: the owner
// threads' stores and the force kernel's loads are coalesced.
#include "device_common.cuh"
#include "kernels.h"

namespace n2p2b
{

namespace
{

constexpr int kSFThreads = 128;
constexpr int kSFWarps = kSFThreads / 32;

// CutoffFunction::fdf for the group's cutoff (type is global in n2p2).
__device__ __forceinline__ void cutoffFdf(SFParams const& P, DevGroup const& g,
                                          double r, double& fc, double& dfc)
{
    if (r >= g.rc)
    {
        fc = 0.0;
        dfc = 0.0;
        return;
    }
    switch (P.cutoffType)
    {
    case 0: // CT_HARD
        fc = 1.0;
        dfc = 0.0;
        return;
    case 1: // CT_COS (fdfCOS)
    {
        if (r < g.rci)
        {
            fc = 1.0;
            dfc = 0.0;
            return;
        }
        double const x = (r - g.rci) * g.iw;
        double const temp = cos(P.PI * x);
        fc = 0.5 * (temp + 1.0);
        dfc = -0.5 * g.iw * P.PI * sqrt(1.0 - temp * temp);
        return;
    }
    case 2: // CT_TANHU
    {
        double const temp = tanh(1.0 - r * g.rcinv);
        double const temp2 = temp * temp;
        fc = temp * temp2;
        dfc = 3.0 * temp2 * (temp2 - 1.0) * g.rcinv;
        return;
    }
    case 3: // CT_TANH
    {
        double const temp = tanh(1.0 - r * g.rcinv);
        double const temp2 = temp * temp;
        fc = P.TANH_PRE * temp * temp2;
        dfc = 3.0 * P.TANH_PRE * temp2 * (temp2 - 1.0) * g.rcinv;
        return;
    }
    default: // CT_EXP, CT_POLY1..4 (fdfCORE with CoreFunction)
    {
        if (r < g.rci)
        {
            fc = 1.0;
            dfc = 0.0;
            return;
        }
        double const x = (r - g.rci) * g.iw;
        double fx, dfx;
        switch (P.cutoffType)
        {
        case 4: // CT_EXP
        {
            double const temp = 1.0 / (x * x - 1.0);
            double const temp2 = exp(temp);
            fx = P.E * temp2;
            dfx = -2.0 * P.E * x * temp * temp * temp2;
            break;
        }
        case 5: // CT_POLY1
            fx = (2.0 * x - 3.0) * x * x + 1.0;
            dfx = x * (6.0 * x - 6.0);
            break;
        case 6: // CT_POLY2
        {
            double const x2 = x * x;
            fx = ((15.0 - 6.0 * x) * x - 10.0) * x * x2 + 1.0;
            dfx = x2 * ((60.0 - 30.0 * x) * x - 30.0);
            break;
        }
        case 7: // CT_POLY3
        {
            double const x2 = x * x;
            fx = (x * (x * (20.0 * x - 70.0) + 84.0) - 35.0) * x2 * x2 + 1.0;
            dfx = x2 * x * (x * (x * (140.0 * x - 420.0) + 420.0) - 140.0);
            break;
        }
        default: // CT_POLY4
        {
            double x4 = x * x;
            x4 *= x4;
            fx = (x * (x * ((315.0 - 70.0 * x) * x - 540.0) + 420.0) - 126.0)
                 * x * x4 + 1.0;
            dfx = x4 * (x * (x * ((2520.0 - 630.0 * x) * x - 3780.0) + 2520.0)
                        - 630.0);
            break;
        }
        }
        fc = fx;
        dfc = dfx * g.iw;
        return;
    }
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

struct SFShared
{
    double* dx;
    double* dy;
    double* dz;
    double* d;
    double* fc;
    double* dfc;
    double* wpG;   // [warp][maxSF]
    double* wpS;   // [warp][maxSF][3]
};

// Adds one member's per-thread partial (G, self) into the warp slot.
__device__ __forceinline__ void flushMember(SFShared const& sh, int maxSF,
                                           int sf, double g, double sx,
                                           double sy, double sz)
{
    g = warpSum(g);
    sx = warpSum(sx);
    sy = warpSum(sy);
    sz = warpSum(sz);
    if ((threadIdx.x & 31) == 0)
    {
        int const w = threadIdx.x >> 5;
        sh.wpG[w * maxSF + sf] += g;
        double* s = sh.wpS + ((long)w * maxSF + sf) * 3;
        s[0] += sx;
        s[1] += sy;
        s[2] += sz;
    }
}

template <int MC>
__device__ void radialGroup(SFParams const& P, DevGroup const& g,
                            SFShared const& sh, int const eb[kMaxElem + 1],
                            int cnt, double* __restrict__ dGdrAtom,
                            int derivatives)
{
    int const e1 = g.e1;
    int const ob = eb[e1];
    int const on = eb[e1 + 1] - ob;
    for (int mb = 0; mb < g.mcnt; mb += MC)
    {
        int const mc = min(MC, g.mcnt - mb);
        for (int o0 = 0; o0 < on; o0 += kSFThreads)
        {
            int const o = o0 + threadIdx.x;
            bool const active = o < on;
            int const t = ob + (active ? o : 0);
            double const r = sh.d[t];
            bool const valid = active && (r < g.rc);
            double const pfc = sh.fc[t];
            double const pdfc = sh.dfc[t];
            double const d1[3] = {sh.dx[t], sh.dy[t], sh.dz[t]};
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                if (l >= mc) break;
                DevMember const& M = P.members[g.mbeg + mb + l];
                double gsum = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
                double v0 = 0.0, v1 = 0.0, v2 = 0.0;
                if (valid)
                {
                    double const rr = r - M.rs;
                    double const pexp = exp(-M.eta * rr * rr);
                    gsum = pexp * pfc;
                    double const p1 = M.factorNorm
                                    * (pdfc - 2.0 * M.eta * rr * pfc)
                                    * pexp / r;
                    sx = p1 * d1[0];
                    sy = p1 * d1[1];
                    sz = p1 * d1[2];
                    v0 = -sx;
                    v1 = -sy;
                    v2 = -sz;
                }
                if (derivatives && active)
                {
                    long const s = M.slot[e1];
                    dGdrAtom[(s * 3 + 0) * cnt + t] = v0;
                    dGdrAtom[(s * 3 + 1) * cnt + t] = v1;
                    dGdrAtom[(s * 3 + 2) * cnt + t] = v2;
                }
                flushMember(sh, P.maxSF, M.sf, gsum, sx, sy, sz);
            }
        }
    }
}

template <int MC, bool NARROW>
__device__ void angularGroup(SFParams const& P, DevGroup const& g,
                             SFShared const& sh, int const eb[kMaxElem + 1],
                             int cnt, double* __restrict__ dGdrAtom,
                             int derivatives)
{
    int const e1 = g.e1;
    int const e2 = g.e2;
    int const b1 = eb[e1], n1 = eb[e1 + 1] - eb[e1];
    int const b2 = eb[e2], n2 = eb[e2 + 1] - eb[e2];
    int const numOwners = (e1 == e2) ? n1 : n1 + n2;
    double const rc = g.rc;
    for (int mb = 0; mb < g.mcnt; mb += MC)
    {
        int const mc = min(MC, g.mcnt - mb);
        for (int o0 = 0; o0 < numOwners; o0 += kSFThreads)
        {
            int const o = o0 + threadIdx.x;
            bool const active = o < numOwners;
            int t, et, pb, pn;
            if (!active || o < n1)
            {
                t = b1 + (active ? o : 0);
                et = e1;
                pb = b2;
                pn = n2;
            }
            else
            {
                t = b2 + (o - n1);
                et = e2;
                pb = b1;
                pn = n1;
            }
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
            double const rij = sh.d[t];
            bool const valid = active && (rij < rc);
            double const dr1[3] = {sh.dx[t], sh.dy[t], sh.dz[t]};
            if (valid)
            {
                double const r2ij = rij * rij;
                double const pfcij = sh.fc[t];
                double const pdfcij = sh.dfc[t];
                double const rc2 = g.rc2;
                for (int k = pb; k < pb + pn; ++k)
                {
                    if (k == t) continue;
                    double const rik = sh.d[k];
                    if (!(rik < rc)) continue;
                    double const dr2[3] = {sh.dx[k], sh.dy[k], sh.dz[k]};
                    double const dr3[3] = {dr2[0] - dr1[0], dr2[1] - dr1[1],
                                           dr2[2] - dr1[2]};
                    double rjk = 0.0, pfcjk = 1.0, pdfcjk = 0.0;
                    if (NARROW)
                    {
                        rjk = dr3[0] * dr3[0] + dr3[1] * dr3[1]
                            + dr3[2] * dr3[2];
                        if (!(rjk < rc2)) continue;
                        rjk = sqrt(rjk);
                        cutoffFdf(P, g, rjk, pfcjk, pdfcjk);
                    }
                    double const pfcik = sh.fc[k];
                    double const rinvijik = 1.0 / rij / rik;
                    double const costijk = (dr1[0] * dr2[0] + dr1[1] * dr2[1]
                                            + dr1[2] * dr2[2]) * rinvijik;
                    double const r2ik = rik * rik;
                    double pfc, r2sum, pr1, pr3 = 0.0;
                    if (NARROW)
                    {
                        pfc = pfcij * pfcik * pfcjk;
                        r2sum = r2ij + r2ik + rjk * rjk;
                        pr1 = pfcik * pfcjk * pdfcij / rij;
                        pr3 = pfcij * pfcik * pdfcjk / rjk;
                    }
                    else
                    {
                        pfc = pfcij * pfcik;
                        r2sum = r2ij + r2ik;
                        pr1 = pfcik * pdfcij / rij;
                    }
                    double const cr = costijk / r2ij;
                    double vexp = 0.0, rijs = 0.0, riks = 0.0, rjks = 0.0;
#pragma unroll
                    for (int l = 0; l < MC; ++l)
                    {
                        if (l >= mc) break;
                        DevMember const& M = P.members[g.mbeg + mb + l];
                        if (M.calcExp)
                        {
                            if (M.rsPositive)
                            {
                                rijs = rij - M.rs;
                                riks = rik - M.rs;
                                if (NARROW)
                                {
                                    rjks = rjk - M.rs;
                                    vexp = exp(-M.eta * (rijs * rijs
                                                         + riks * riks
                                                         + rjks * rjks));
                                }
                                else
                                {
                                    vexp = exp(-M.eta * (rijs * rijs
                                                         + riks * riks));
                                }
                            }
                            else
                            {
                                vexp = exp(-M.eta * r2sum);
                            }
                        }
                        double const plambda = 1.0 + M.lambda * costijk;
                        double fg = vexp;
                        if (plambda <= 0.0) fg = 0.0;
                        else if (M.useIntPow)
                            fg *= powInt(plambda, M.zetaInt - 1);
                        else
                            fg *= pow(plambda, M.zeta - 1.0);
                        aG[l] += fg * plambda * pfc;
                        fg *= M.factorNorm;
                        double const pfczl = pfc * M.zetaLambda;
                        double const p2etapl = plambda * M.factorDeriv;
                        double p1, p3;
                        if (M.rsPositive)
                        {
                            p1 = fg * (pfczl * (rinvijik - cr
                                                - p2etapl * rijs / rij)
                                       + pr1 * plambda);
                            if (NARROW)
                                p3 = fg * (pfczl * (rinvijik
                                                    + p2etapl * rjks / rjk)
                                           - pr3 * plambda);
                            else
                                p3 = fg * pfczl * rinvijik;
                        }
                        else
                        {
                            p1 = fg * (pfczl * (rinvijik - cr - p2etapl)
                                       + pr1 * plambda);
                            if (NARROW)
                                p3 = fg * (pfczl * (rinvijik + p2etapl)
                                           - pr3 * plambda);
                            else
                                p3 = fg * pfczl * rinvijik;
                        }
                        aP1[l] += p1;
                        aPx[l] += p3 * dr3[0];
                        aPy[l] += p3 * dr3[1];
                        aPz[l] += p3 * dr3[2];
                    }
                }
            }
#pragma unroll
            for (int l = 0; l < MC; ++l)
            {
                if (l >= mc) break;
                DevMember const& M = P.members[g.mbeg + mb + l];
                double const sx = aP1[l] * dr1[0];
                double const sy = aP1[l] * dr1[1];
                double const sz = aP1[l] * dr1[2];
                if (derivatives && active)
                {
                    long const s = M.slot[et];
                    dGdrAtom[(s * 3 + 0) * cnt + t] = -(sx + aPx[l]);
                    dGdrAtom[(s * 3 + 1) * cnt + t] = -(sy + aPy[l]);
                    dGdrAtom[(s * 3 + 2) * cnt + t] = -(sz + aPz[l]);
                }
                flushMember(sh, P.maxSF, M.sf, 0.5 * aG[l], sx, sy, sz);
            }
        }
    }
}

template <int MC>
__global__ void __launch_bounds__(kSFThreads)
sfFp64Kernel(__grid_constant__ SFParams const P, SFLaunch const L)
{
    extern __shared__ double smem[];
    int const cap = L.cap;
    int const maxSF = P.maxSF;
    SFShared sh;
    sh.dx = smem;
    sh.dy = sh.dx + cap;
    sh.dz = sh.dy + cap;
    sh.d = sh.dz + cap;
    sh.fc = sh.d + cap;
    sh.dfc = sh.fc + cap;
    sh.wpG = sh.dfc + cap;
    sh.wpS = sh.wpG + kSFWarps * maxSF;
    int const numElements = P.numElements;

    for (int i = blockIdx.x; i < L.n; i += gridDim.x)
    {
        if (L.status[ST_FLAGS] & FLAG_ABORT) return;
        int const ec = L.elem[i];
        long const beg = L.nbrOff[i];
        int const cnt = L.nbrOff[i + 1] - (int)beg;
        if (cnt > cap)
        {
            if (threadIdx.x == 0)
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
        for (int t = threadIdx.x; t < cnt; t += kSFThreads)
        {
            sh.dx[t] = L.dx[beg + t];
            sh.dy[t] = L.dy[beg + t];
            sh.dz[t] = L.dz[beg + t];
            sh.d[t] = L.dd[beg + t];
        }
        for (int k = threadIdx.x; k < kSFWarps * maxSF * 4; k += kSFThreads)
            sh.wpG[k] = 0.0;  // wpG and wpS are contiguous
        double* dGdrAtom = L.dGdr + beg * (long)P.maxSlots * 3;
        double lastRc = -1.0;
        for (int gi = P.groupBeg[ec]; gi < P.groupBeg[ec + 1]; ++gi)
        {
            DevGroup const& g = P.groups[gi];
            if (g.rc != lastRc)
            {
                __syncthreads();
                for (int t = threadIdx.x; t < cnt; t += kSFThreads)
                {
                    double fc, dfc;
                    cutoffFdf(P, g, sh.d[t], fc, dfc);
                    sh.fc[t] = fc;
                    sh.dfc[t] = dfc;
                }
                lastRc = g.rc;
                __syncthreads();
            }
            if (g.type == 2)
                radialGroup<MC>(P, g, sh, eb, cnt, dGdrAtom, L.derivatives);
            else if (g.type == 3)
                angularGroup<MC, true>(P, g, sh, eb, cnt, dGdrAtom,
                                       L.derivatives);
            else
                angularGroup<MC, false>(P, g, sh, eb, cnt, dGdrAtom,
                                        L.derivatives);
        }
        __syncthreads();
        int const nsf = P.numSF[ec];
        SFScale const* sc = L.scale + (long)ec * maxSF;
        for (int s = threadIdx.x; s < nsf; s += kSFThreads)
        {
            double raw = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
            for (int w = 0; w < kSFWarps; ++w)
            {
                raw += sh.wpG[w * maxSF + s];
                double const* p = sh.wpS + ((long)w * maxSF + s) * 3;
                sx += p[0];
                sy += p[1];
                sz += p[2];
            }
            SFScale const q = sc[s];
            L.G[(long)i * maxSF + s] = q.smin + q.b * (q.q * raw - q.shift);
            if (L.derivatives)
            {
                double* o = L.dGdrSelf + ((long)i * maxSF + s) * 3;
                o[0] = sx;
                o[1] = sy;
                o[2] = sz;
            }
        }
        __syncthreads();
    }
}

} // namespace

std::size_t sfSharedBytes(SFParams const& P, int cap)
{
    return sizeof(double) * ((std::size_t)6 * cap
                             + (std::size_t)kSFWarps * P.maxSF * 4);
}

int sfBlocksPerSM(SFParams const& P, int cap)
{
    std::size_t const shm = sfSharedBytes(P, cap);
    cudaFuncSetAttribute(sfFp64Kernel<12>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)shm);
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &blocks, sfFp64Kernel<12>, kSFThreads, shm) != cudaSuccess
        || blocks < 1)
        blocks = 1;
    return blocks;
}

void launchSymmetryFunctions(SFParams const& P, SFLaunch const& L,
                             cudaStream_t s)
{
    std::size_t const shm = sfSharedBytes(P, L.cap);
    if (L.memberChunk <= 8)
    {
        cudaFuncSetAttribute(sfFp64Kernel<8>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)shm);
        sfFp64Kernel<8><<<L.grid, kSFThreads, shm, s>>>(P, L);
    }
    else
    {
        cudaFuncSetAttribute(sfFp64Kernel<12>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)shm);
        sfFp64Kernel<12><<<L.grid, kSFThreads, shm, s>>>(P, L);
    }
}

} // namespace n2p2b
