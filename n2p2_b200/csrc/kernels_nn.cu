// Atomic neural networks, forces and energy (FP64 plain form).
//
// NN: NeuralNetwork::propagate / propagateLayer (libnnp/NeuralNetwork.cpp:
// 386-394, 761-896) and NeuralNetwork::calculateDEdG (:396-442).  The
// reference computes dE/dG in forward mode, one input at a time; here it is
// the reverse-mode sweep (one backward pass of the single output), the same
// derivative up to summation order.  One warp per atom, lanes over neurons;
// W^T (in-major) for the forward sweep and W (out-major) for the backward
// sweep so both read coalesced rows.
//
// Forces: Mode::calculateForces (libnnp/Mode.cpp:1849-1912) with
// Atom::calculateSelfForceShort / calculatePairForceShort (libnnp/Atom.cpp:
// 371-401).  The reference gathers, for atom i, the pair terms of every entry
// (j -> i) in the lists of i's unique neighbors j != i.  By list symmetry
// those entries are exactly the mirrors of i's own entries (i -> j, bc), so:
//   pass 1 (warp per owner atom j, lanes over its entries, coalesced reads
//           of the stored dG/dr):  pairF[e] = -sum_s dEdG_j[table(s)] dGdr[e][s]
//           and selfF[j] = -sum_s dEdG_j[s] dGdr_self[j][s] = -sum_e pairF[e]
//           (the reference's self derivative is minus the sum of the
//           neighbor slots: SymGrpExpRad.cpp:215-226,
//           SymGrpExpAngn.cpp:366-383);
//   pass 2 (thread per atom i): F_i = selfF_i + sum over i's entries e with
//           index != i of pairF[mirror[e]]
// -- a fixed-order segmented reduction, no atomics.  Entries of i pointing to
// i itself (periodic self-images) are skipped exactly as the reference skips
// i in neighborsUnique.
#include "device_common.cuh"
#include "kernels.h"

namespace n2p2b
{

namespace
{

constexpr int kNNWarps = 4;
constexpr int kPairChunks = 4;      // entries per lane in one pair-force block
constexpr int kPairAhead = 4;       // slots prefetched ahead into L2
constexpr double kExpLimit = 35.0;  // EXP_LIMIT, libnnp/NeuralNetwork.cpp:25

// Activation value and derivative (NeuralNetwork::propagateLayer).
__device__ __forceinline__ void activate(int a, double x, double& v,
                                         double& dv)
{
    switch (a)
    {
    case 0: // AF_IDENTITY
        v = x;
        dv = 1.0;
        return;
    case 1: // AF_TANH
    {
        double const t = tanh(x);
        v = t;
        dv = 1.0 - t * t;
        return;
    }
    case 2: // AF_LOGISTIC
        if (x > kExpLimit) { v = 1.0; dv = 0.0; return; }
        if (x < -kExpLimit) { v = 0.0; dv = 0.0; return; }
        {
            double const t = 1.0 / (1.0 + exp(-x));
            v = t;
            dv = t * (1.0 - t);
        }
        return;
    case 3: // AF_SOFTPLUS
        if (x > kExpLimit) { v = x; dv = 1.0; return; }
        if (x < -kExpLimit) { v = 0.0; dv = 0.0; return; }
        {
            double const t = exp(x);
            v = log(1.0 + t);
            dv = 1.0 / (1.0 + 1.0 / t);
        }
        return;
    case 4: // AF_RELU
        if (x > 0.0) { v = x; dv = 1.0; }
        else { v = 0.0; dv = 0.0; }
        return;
    case 5: // AF_GAUSSIAN
    {
        double const t = exp(-0.5 * x * x);
        v = t;
        dv = -x * t;
        return;
    }
    case 6: // AF_COS
        v = cos(x);
        dv = -sin(x);
        return;
    case 7: // AF_REVLOGISTIC
    {
        double const t = 1.0 / (1.0 + exp(-x));
        v = 1.0 - t;
        dv = t * (t - 1.0);
        return;
    }
    case 8: // AF_EXP
    {
        double const t = exp(-x);
        v = t;
        dv = -t;
        return;
    }
    default: // AF_HARMONIC
        v = x * x;
        dv = 2.0 * x;
        return;
    }
}

__device__ __forceinline__ void activate(int a, float x, float& v, float& dv)
{
    float const lim = (float)kExpLimit;
    switch (a)
    {
    case 0: v = x; dv = 1.0f; return;
    case 1: { float const t = tanhf(x); v = t; dv = 1.0f - t * t; return; }
    case 2:
        if (x > lim) { v = 1.0f; dv = 0.0f; return; }
        if (x < -lim) { v = 0.0f; dv = 0.0f; return; }
        { float const t = 1.0f / (1.0f + expf(-x)); v = t; dv = t * (1.0f - t); }
        return;
    case 3:
        if (x > lim) { v = x; dv = 1.0f; return; }
        if (x < -lim) { v = 0.0f; dv = 0.0f; return; }
        { float const t = expf(x); v = log1pf(t); dv = 1.0f / (1.0f + 1.0f / t); }
        return;
    case 4:
        if (x > 0.0f) { v = x; dv = 1.0f; } else { v = 0.0f; dv = 0.0f; }
        return;
    case 5: { float const t = expf(-0.5f * x * x); v = t; dv = -x * t; return; }
    case 6: v = cosf(x); dv = -sinf(x); return;
    case 7:
    { float const t = 1.0f / (1.0f + expf(-x)); v = 1.0f - t; dv = t * (t - 1.0f);
      return; }
    case 8: { float const t = expf(-x); v = t; dv = -t; return; }
    default: v = x * x; dv = 2.0f * x; return;
    }
}

// Warp per atom.  Shared memory per warp: activations of the current layer
// (maxWidth) and the activation derivatives of every layer (L * maxWidth).
// T = double: the plain form; T = float: the distilled student network.
template <typename T>
__global__ void __launch_bounds__(32 * kNNWarps)
nnKernel(__grid_constant__ NNParams const P, NNLaunch const L)
{
    extern __shared__ double smemD[];
    T* const smem = reinterpret_cast<T*>(smemD);
    T const* const weights = static_cast<T const*>(L.weights);
    T const* const Gin = static_cast<T const*>(L.G);
    T* const dEdGout = static_cast<T*>(L.dEdG);
    int const lane = threadIdx.x & 31;
    int const w = threadIdx.x >> 5;
    int const W = P.maxWidth;
    T* x = smem + (long)w * W * (kMaxLayers + 2);
    T* y = x + W;
    T* dfs = y + W;  // [layer][W]
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;
    for (int i = blockIdx.x * kNNWarps + w; i < L.n;
         i += gridDim.x * kNNWarps)
    {
        int const e = L.elem[i];
        int const nl = P.numLayers[e];
        int const nin = P.width[e][0];
        T const* g = Gin + (long)i * L.maxSF;
        for (int k = lane; k < nin; k += 32) x[k] = g[k];
        __syncwarp();
        T out = T(0);
        for (int l = 1; l < nl; ++l)
        {
            int const ni = P.width[e][l - 1];
            int const no = P.width[e][l];
            T const* Wt = weights + P.wtoff[e][l];
            T const* b = weights + P.boff[e][l];
            int const act = P.act[e][l];
            for (int o = lane; o < no; o += 32)
            {
                T acc = T(0);
                for (int j = 0; j < ni; ++j) acc += Wt[(long)j * no + o] * x[j];
                acc += b[o];
                if (P.normalizeNeurons) acc /= ni;
                T v, dv;
                activate(act, acc, v, dv);
                y[o] = v;
                dfs[l * W + o] = dv;
            }
            __syncwarp();
            for (int o = lane; o < no; o += 32) x[o] = y[o];
            __syncwarp();
        }
        out = x[0];
        if (lane == 0) L.energy[i] = (double)out;
        if (L.derivatives)
        {
            // delta_L = f'_L (/ n_{L-1}); delta_{l-1}[j] =
            //   f'_{l-1}[j] * sum_o W_l[o][j] delta_l[o] (/ n_{l-2})
            int const nlast = P.width[e][nl - 2];
            T* d = y;  // delta of the current layer
            if (lane == 0)
            {
                T v = dfs[(nl - 1) * W + 0];
                if (P.normalizeNeurons) v /= nlast;
                d[0] = v;
            }
            __syncwarp();
            for (int l = nl - 1; l >= 1; --l)
            {
                int const ni = P.width[e][l - 1];
                int const no = P.width[e][l];
                T const* Wm = weights + P.woff[e][l];
                for (int j = lane; j < ni; j += 32)
                {
                    T acc = T(0);
                    for (int o = 0; o < no; ++o)
                        acc += Wm[(long)o * ni + j] * d[o];
                    if (l > 1)
                    {
                        acc *= dfs[(l - 1) * W + j];
                        if (P.normalizeNeurons) acc /= P.width[e][l - 2];
                    }
                    x[j] = acc;
                }
                __syncwarp();
                for (int j = lane; j < ni; j += 32) d[j] = x[j];
                __syncwarp();
            }
            T* o = dEdGout + (long)i * L.maxSF;
            for (int k = lane; k < nin; k += 32) o[k] = d[k];
        }
        __syncwarp();
    }
}

// Pass 1: warp per owner atom j.  T is the type of dE/dG and dG/dr (double,
// or float in the mixed form); products and sums are formed in FP64.
template <typename T>
__global__ void __launch_bounds__(128)
pairForceKernel(ForceLaunch const L)
{
    extern __shared__ double smem[];
    int const lane = threadIdx.x & 31;
    int const w = threadIdx.x >> 5;
    int const warps = blockDim.x >> 5;
    int const S = L.maxSlots;
    // dE/dG of the owner, then its coefficients per (neighbor element, slot)
    // so the entry loop reads one shared word per slot.
    double* dE = smem + (long)w * (L.maxSF + L.numElements * S);
    double* cE = dE + L.maxSF;
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;
    T const* const dEdG = static_cast<T const*>(L.dEdG);
    T const* const dGdr = static_cast<T const*>(L.dGdr);
    for (int j = blockIdx.x * warps + w; j < L.n; j += gridDim.x * warps)
    {
        int const ej = L.elem[j];
        T const* src = dEdG + (long)j * L.maxSF;
        for (int s = lane; s < L.maxSF; s += 32) dE[s] = (double)src[s];
        __syncwarp();
        for (int k = lane; k < L.numElements * S; k += 32)
        {
            int const en = k / S, s = k - en * S;
            cE[k] = s < L.numSlots[ej][en]
                  ? dE[L.slotSF[((long)ej * kMaxElem + en) * S + s]] : 0.0;
        }
        __syncwarp();
        // Pair terms of j's entries; the self force is minus their sum.
        // Blocks of 32 * kPairChunks entries, slot loop outermost: the warp
        // reads each (slot, component) row of the block as one contiguous
        // run, so no DRAM sector is fetched twice.
        double fx = 0.0, fy = 0.0, fz = 0.0;
        long const b = L.nbrOff[j];
        int const cnt = L.nbrOff[j + 1] - (int)b;
        T const* gd = dGdr + b * (long)S * 3;
        int smax = 0;
        for (int en = 0; en < L.numElements; ++en)
            smax = max(smax, L.numSlots[ej][en]);
        for (int t0 = 0; t0 < cnt; t0 += 32 * kPairChunks)
        {
            double px[kPairChunks], py[kPairChunks], pz[kPairChunks];
            int ns[kPairChunks], eo[kPairChunks];
#pragma unroll
            for (int k = 0; k < kPairChunks; ++k)
            {
                int const t = t0 + 32 * k + lane;
                int const en = t < cnt ? L.nbrEl[b + t] : 0;
                ns[k] = t < cnt ? L.numSlots[ej][en] : 0;
                eo[k] = en * S;
                px[k] = py[k] = pz[k] = 0.0;
            }
            for (int s = 0; s < smax; ++s)
            {
                // Lanes 0-2 ask L2 for the three component rows of slot
                // s + kPairAhead (their 16-byte-aligned inner part, inside
                // the atom's block), so the loads of later slots find them
                // there.
                if (lane < 3 && s + kPairAhead < smax)
                {
                    T const* r = gd + ((long)(s + kPairAhead) * 3 + lane) * cnt;
                    unsigned long long const a =
                        (reinterpret_cast<unsigned long long>(r + t0) + 15)
                        & ~15ull;
                    unsigned long long const e =
                        reinterpret_cast<unsigned long long>(
                            r + min(cnt, t0 + 32 * kPairChunks)) & ~15ull;
                    if (e > a)
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                                     :: "l"(a), "r"((unsigned)(e - a))
                                     : "memory");
                }
                T const* row = gd + (long)s * 3 * cnt + t0 + lane;
#pragma unroll
                for (int k = 0; k < kPairChunks; ++k)
                    if (s < ns[k])
                    {
                        double const c = cE[eo[k] + s];
                        T const* g = row + 32 * k;
                        px[k] -= c * (double)g[0];
                        py[k] -= c * (double)g[cnt];
                        pz[k] -= c * (double)g[2 * cnt];
                    }
            }
#pragma unroll
            for (int k = 0; k < kPairChunks; ++k)
            {
                int const t = t0 + 32 * k + lane;
                if (t >= cnt) continue;
                L.pairF[(b + t) * 3 + 0] = px[k];
                L.pairF[(b + t) * 3 + 1] = py[k];
                L.pairF[(b + t) * 3 + 2] = pz[k];
                fx -= px[k];
                fy -= py[k];
                fz -= pz[k];
            }
        }
        fx = warpSum(fx);
        fy = warpSum(fy);
        fz = warpSum(fz);
        if (lane == 0)
        {
            L.selfF[(long)j * 3 + 0] = fx;
            L.selfF[(long)j * 3 + 1] = fy;
            L.selfF[(long)j * 3 + 2] = fz;
        }
        __syncwarp();
    }
}

// Warp per atom j: dG/dr_j (self) = -sum over j's entries of the slots,
// neighbor element by neighbor element, lanes over entries.
template <typename T>
__global__ void __launch_bounds__(128)
selfDerivativeKernel(ForceLaunch const L, T* __restrict__ out)
{
    extern __shared__ double acc0[];
    int const lane = threadIdx.x & 31;
    int const w = threadIdx.x >> 5;
    int const warps = blockDim.x >> 5;
    double* acc = acc0 + (long)w * L.maxSF * 3;
    T const* const dGdr = static_cast<T const*>(L.dGdr);
    for (int j = blockIdx.x * warps + w; j < L.n; j += gridDim.x * warps)
    {
        int const ej = L.elem[j];
        for (int k = lane; k < L.maxSF * 3; k += 32) acc[k] = 0.0;
        __syncwarp();
        long const b = L.nbrOff[j];
        int const cnt = L.nbrOff[j + 1] - (int)b;
        T const* gd = dGdr + b * (long)L.maxSlots * 3;
        for (int en = 0; en < L.numElements; ++en)
        {
            int16_t const* tab = L.slotSF + ((long)ej * kMaxElem + en)
                                            * L.maxSlots;
            for (int sl = 0; sl < L.numSlots[ej][en]; ++sl)
                for (int c = 0; c < 3; ++c)
                {
                    double v = 0.0;
                    for (int t = lane; t < cnt; t += 32)
                        if (L.nbrEl[b + t] == en)
                            v += (double)gd[((long)sl * 3 + c) * cnt + t];
                    v = warpSum(v);
                    if (lane == 0) acc[tab[sl] * 3 + c] -= v;
                    __syncwarp();
                }
        }
        for (int k = lane; k < L.maxSF * 3; k += 32)
            out[(long)j * L.maxSF * 3 + k] = (T)acc[k];
        __syncwarp();
    }
}

// Pass 2: warp per atom.  Lane l sums the mirror pair terms of entries
// l, l + 32, ... of the atom in that order, then a fixed butterfly adds the
// lanes' partial sums, so every run adds in the same order (deterministic)
// while the 32 lanes' gathers are in flight together.
__global__ void __launch_bounds__(256)
gatherForceKernel(ForceLaunch const L)
{
    int const lane = threadIdx.x & 31;
    long const i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= L.n) return;
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    int const eb = L.nbrOff[i], ee = L.nbrOff[i + 1];
    for (int e = eb + lane; e < ee; e += 32)
    {
        if (L.nbrIdx[e] == i) continue;
        long const m = L.mirror[e];
        if (m < 0) continue;  // flagged by the mirror kernel; never read OOB
        fx += L.pairF[m * 3 + 0];
        fy += L.pairF[m * 3 + 1];
        fz += L.pairF[m * 3 + 2];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (lane != 0) return;
    fx += L.selfF[i * 3 + 0];
    fy += L.selfF[i * 3 + 1];
    fz += L.selfF[i * 3 + 2];
    // Atom::toPhysicalUnits: f /= convEnergy / convLength.
    L.F[i * 3 + 0] = fx / L.forceScale;
    L.F[i * 3 + 1] = fy / L.forceScale;
    L.F[i * 3 + 2] = fz / L.forceScale;
}

// Deterministic energy sum (fixed tree) + Structure::toPhysicalUnits +
// Mode::addEnergyOffset (libnnp/Mode.cpp:2018-2035).
__global__ void energyKernel(EnergyLaunch const L)
{
    __shared__ double part[1024];
    int const t = threadIdx.x;
    double s = 0.0;
    for (int i = t; i < L.n; i += blockDim.x) s += L.atomicEnergy[i];
    part[t] = s;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1)
    {
        if (t < h) part[t] += part[t + h];
        __syncthreads();
    }
    if (t == 0)
    {
        double const en = part[0];
        double e = en;
        if (L.normalize)
            e = e / L.convEnergy + (double)L.n * L.meanEnergy;
        for (int k = 0; k < L.numElements; ++k) e += L.offsetTerm[k];
        L.out[0] = en;
        L.out[1] = e;
    }
}

// Block per structure of a batch: the energy kernel's fixed tree over the
// structure's atoms, then Structure::toPhysicalUnits and
// Mode::addEnergyOffset for that structure.
__global__ void energyBatchKernel(BatchEnergyLaunch const L)
{
    __shared__ double part[256];
    int const s = blockIdx.x;
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;
    BatchStruct const& B = L.bs[s];
    int const t = threadIdx.x;
    double v = 0.0;
    for (int i = B.atomBeg + t; i < B.atomEnd; i += blockDim.x)
        v += L.atomicEnergy[i];
    part[t] = v;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1)
    {
        if (t < h) part[t] += part[t + h];
        __syncthreads();
    }
    if (t == 0)
    {
        double e = part[0];
        if (L.normalize)
            e = e / L.convEnergy
              + (double)(B.atomEnd - B.atomBeg) * L.meanEnergy;
        for (int k = 0; k < L.numElements; ++k)
            e += (double)(B.es[k + 1] - B.es[k]) * L.offset[k];
        L.out[s] = e;
    }
}

__global__ void __launch_bounds__(256)
targetForceKernel(TargetForceLaunch const L)
{
    // Warp per target: lane l sums reverse entries l, l + 32, ... in that
    // order, a fixed butterfly adds the lanes (deterministic).
    int const lane = threadIdx.x & 31;
    long const m = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (m >= L.numTargets) return;
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int k = L.revOff[m] + lane; k < L.revOff[m + 1]; k += 32)
    {
        long const e = L.revEntry[k];
        fx += L.pairF[e * 3 + 0];
        fy += L.pairF[e * 3 + 1];
        fz += L.pairF[e * 3 + 2];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (lane != 0) return;
    if (m < L.numLocal)
    {
        fx += L.selfF[m * 3 + 0];
        fy += L.selfF[m * 3 + 1];
        fz += L.selfF[m * 3 + 2];
    }
    L.F[m * 3 + 0] = fx / L.forceScale;
    L.F[m * 3 + 1] = fy / L.forceScale;
    L.F[m * 3 + 2] = fz / L.forceScale;
}

} // namespace

void launchTargetForces(TargetForceLaunch const& L, cudaStream_t s)
{
    int const tb = 256;    // 8 targets (warps) per block
    long const g = ((long)L.numTargets * 32 + tb - 1) / tb;
    noteLaunches(1);
    targetForceKernel<<<g > 0 ? (int)g : 1, tb, 0, s>>>(L);
}

void launchEnergyBatch(BatchEnergyLaunch const& L, cudaStream_t s)
{
    noteLaunches(1);
    energyBatchKernel<<<L.numStructs > 0 ? L.numStructs : 1, 256, 0, s>>>(L);
}

void launchNeuralNetworks(NNParams const& P, NNLaunch const& L,
                          cudaStream_t s)
{
    bool const f = L.precision != PREC_FP64;
    std::size_t const shm = (f ? sizeof(float) : sizeof(double))
                          * (std::size_t)kNNWarps * P.maxWidth
                          * (kMaxLayers + 2);
    int const grid = (L.n + kNNWarps - 1) / kNNWarps;
    noteLaunches(1);
    if (f)
    {
        cudaFuncSetAttribute(nnKernel<float>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)shm);
        nnKernel<float><<<grid > 0 ? grid : 1, 32 * kNNWarps, shm, s>>>(P, L);
    }
    else
    {
        cudaFuncSetAttribute(nnKernel<double>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)shm);
        nnKernel<double><<<grid > 0 ? grid : 1, 32 * kNNWarps, shm, s>>>(P,
                                                                         L);
    }
}

void launchForces(ForceLaunch const& L, cudaStream_t s)
{
    int const warps = 4;
    std::size_t const shm = sizeof(double) * warps
                          * (std::size_t)(L.maxSF + L.numElements * L.maxSlots);
    int const grid = (L.n + warps - 1) / warps;
    noteLaunches(L.gather ? 2 : 1);
    if (L.precision != PREC_FP64)
        pairForceKernel<float><<<grid > 0 ? grid : 1, 32 * warps, shm, s>>>(L);
    else
        pairForceKernel<double><<<grid > 0 ? grid : 1, 32 * warps, shm, s>>>(L);
    if (!L.gather) return;
    int const tb = 256;    // 8 atoms (warps) per block
    long const gb = ((long)L.n * 32 + tb - 1) / tb;
    gatherForceKernel<<<gb > 0 ? (int)gb : 1, tb,
                        0, s>>>(L);
}

void launchSelfDerivatives(ForceLaunch const& L, void* out, cudaStream_t s)
{
    int const warps = 4;
    std::size_t const shm = sizeof(double) * warps * 3 * (std::size_t)L.maxSF;
    int const grid = (L.n + warps - 1) / warps;
    noteLaunches(1);
    if (L.precision != PREC_FP64)
        selfDerivativeKernel<float><<<grid > 0 ? grid : 1, 32 * warps, shm,
                                      s>>>(L, static_cast<float*>(out));
    else
        selfDerivativeKernel<double><<<grid > 0 ? grid : 1, 32 * warps, shm,
                                       s>>>(L, static_cast<double*>(out));
}

void launchEnergy(EnergyLaunch const& L, cudaStream_t s)
{
    noteLaunches(1);
    energyKernel<<<1, 1024, 0, s>>>(L);
}

} // namespace n2p2b
