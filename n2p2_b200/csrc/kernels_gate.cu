// Extrapolation test on symmetry functions: Element::
// updateSymmetryFunctionStatistics (libnnp/Element.cpp:462-541).
//
// For every atom and each of its element's symmetry functions, the scaled
// value G is mapped back to the raw value with SymFnc::unscale
// (libnnp/SymFnc.cpp:197-223) -- (G - Smin) / scalingFactor + shift, with
// shift = Gmin (ST_SCALE) or Gmean (ST_CENTER, ST_SCALECENTER, ST_SCALESIGMA)
// and (Smin, scalingFactor) = (0, 1) where the type does not scale -- and
// counted as an extrapolation warning when
//     value + eps < lo  or  value - eps > hi,      eps = 1000 DBL_EPSILON,
// the reference's test against the scaling.data range [Gmin, Gmax].  The
// same kernel gates the distilled student network with the student's own
// training range as [lo, hi]: atoms with any warning are appended to
// per-element lists that the teacher network then re-evaluates.
//
// One warp per atom, lanes over symmetry functions; per-atom counts, the
// total in the status words, list order is arbitrary (each listed atom is
// evaluated independently, so results do not depend on it).
#include <cfloat>

#include "device_common.cuh"
#include "kernels.h"

namespace n2p2b
{

namespace
{

template <typename T>
__global__ void __launch_bounds__(128)
ewKernel(EWLaunch const L)
{
    int const lane = threadIdx.x & 31;
    int const warps = blockDim.x >> 5;
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;
    T const* const G = static_cast<T const*>(L.G);
    double const eps = 1000.0 * DBL_EPSILON;
    for (int i = blockIdx.x * warps + (threadIdx.x >> 5); i < L.n;
         i += gridDim.x * warps)
    {
        int const e = L.elem[i];
        int const ns = L.numSF[e];
        int cnt = 0;
        for (int s = lane; s < ns; s += 32)
        {
            SFScale const q = L.scale[(long)e * L.maxSF + s];
            Range const rg = L.range[(long)e * L.maxSF + s];
            double const g = (double)G[(long)i * L.maxSF + s];
            double const value = (g - q.smin) / q.b + q.shift;
            if (value + eps < rg.lo || value - eps > rg.hi) ++cnt;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0)
        {
            if (L.perAtom) L.perAtom[i] = cnt;
            if (cnt > 0)
            {
                atomicAdd(&L.status[L.countSlot], cnt);
                if (L.list)
                {
                    int const pos = atomicAdd(&L.listCount[e], 1);
                    L.list[L.listStart[e] + pos] = i;
                }
            }
        }
    }
}

} // namespace

void launchExtrapolationCheck(EWLaunch const& L, cudaStream_t s)
{
    int const warps = 4;
    int const grid = (L.n + warps - 1) / warps;
    noteLaunches(1);
    if (L.precision != PREC_FP64)
        ewKernel<float><<<grid > 0 ? grid : 1, 32 * warps, 0, s>>>(L);
    else
        ewKernel<double><<<grid > 0 ? grid : 1, 32 * warps, 0, s>>>(L);
}

} // namespace n2p2b
