// Atomic neural networks on the 5th-generation tensor cores (mixed form):
// NeuralNetwork::propagate (libnnp/NeuralNetwork.cpp:386-394, 761-896) and
// NeuralNetwork::calculateDEdG (:396-442) for 128 atoms of one element at a
// time.
//
// One CTA (4 warps, persistent over tiles) per SM.  Per tile:
//   forward   z_l = W_l h_{l-1} + b_l   as D[128 x out] = A[128 x in] B^T with
//             B = W_l (out x in, K-major), one tcgen05.mma per 16 of K;
//   output    E = f_out(w . h_H + b)    FP32 dot product in the epilogue;
//   backward  delta_H = f_out' w * f_H'; delta_{l-1} = (W_l^T delta_l) * f_{l-1}'
//             dE/dG = W_1^T delta_1     as GEMMs with B = W_l^T (in x out).
// Operands are BF16 in shared memory in the UMMA canonical K-major layout
// without swizzle (8-row x 16-byte core matrices; LBO = 128 B between the
// two K halves of an MMA step, SBO = K * 16 B between 8-row groups);
// accumulators are FP32 in tensor memory (row = lane, column = neuron).
// Thread r of the CTA owns row (atom) r: it reads its accumulator row with
// tcgen05.ld, applies bias and activation in FP32, keeps f' in shared memory
// for the backward sweep and writes the next layer's BF16 operand row.
// One elected thread issues the MMAs and commits them to an mbarrier; every
// wait is bounded and reports FLAG_TC_TIMEOUT instead of hanging.
//
// The weights are laid out by the host (tcBuild) so that a CTA copies an
// element's whole weight region into shared memory with 16-byte loads.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "kernels.h"

namespace n2p2b
{

namespace
{

constexpr int kTcThreads = 128;
constexpr long kWaitLimit = 1L << 22;     // try_wait rounds before giving up
constexpr float kExpLimitF = 35.0f;       // EXP_LIMIT, NeuralNetwork.cpp:25

struct TcSmemLayout
{
    int offF, offAh, offAl, offBar, total;
};

// Shared memory: the current element's weights (BF16 high and low parts of
// W and W^T per hidden layer), its FP32 biases and output weights, one
// operand tile of 128 rows (high and low parts; each GEMM's epilogue
// overwrites it in place with the next GEMM's operand once the GEMM has
// completed), and the mbarrier / tensor-memory address words.
__host__ __device__ inline TcSmemLayout tcLayout(TcNNParams const& P)
{
    TcSmemLayout s;
    s.offF = P.wMax;
    int a = s.offF + 4 * P.fMax;
    a = (a + 127) / 128 * 128;
    s.offAh = a;
    a += kTcRows * P.maxP * 2;
    s.offAl = a;
    if (P.split) a += kTcRows * P.maxP * 2;
    s.offBar = a;
    a += 16;
    s.total = a;
    return s;
}

// Byte offset of element (row r, column k) in a K-major operand tile with
// kP columns: core matrix (r / 8, k / 8) of 8 rows x 16 bytes.
__host__ __device__ inline int aOff(int r, int k, int kP)
{
    return (r >> 3) * (kP * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smemAddr(void const* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t ummaDesc(uint32_t addr, uint32_t lbo,
                                             uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu)
         | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16)
         | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32)
         | (1ull << 46);
}

// Instruction descriptor of kind::f16: D = F32, A = B = BF16, both K-major,
// M = 128, N = n.
__device__ __forceinline__ uint32_t idescBF16(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10)
         | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void mmaBF16(uint32_t d, uint64_t a, uint64_t b,
                                        uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n"
        :
        : "r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mmaCommit(uint32_t bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64"
        " [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void tcFenceBefore()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tcFenceAfter()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void proxyFence()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void barInit(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                 :: "r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool barTryWait(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done) : "r"(bar), "r"(parity) : "memory");
    return done != 0;
}

__device__ __forceinline__ bool barWait(uint32_t bar, uint32_t parity)
{
    for (long it = 0; it < kWaitLimit; ++it)
        if (barTryWait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tmemLd16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, "
        "%8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
          "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void tmemSt16(uint32_t taddr, float const v[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, "
        "%9, %10, %11, %12, %13, %14, %15, %16};"
        :: "r"(taddr),
           "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])),
           "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
           "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
           "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
           "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])),
           "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
           "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
           "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}

__device__ __forceinline__ void tmemWaitSt()
{
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// 16 consecutive columns [c0, c0 + 16) of row r (c0 % 16 == 0) as BF16:
// high parts into `hi`, and with `lo` the rounding remainders v - hi.
__device__ __forceinline__ void store16(unsigned char* hi, unsigned char* lo,
                                        int r, int c0, int kP,
                                        float const v[16])
{
    uint32_t wh[8], wl[8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
    {
        __nv_bfloat162 const h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
        wh[q] = *reinterpret_cast<uint32_t const*>(&h);
        float2 const hf = __bfloat1622float2(h);
        __nv_bfloat162 const l = __floats2bfloat162_rn(v[2 * q] - hf.x,
                                                       v[2 * q + 1] - hf.y);
        wl[q] = *reinterpret_cast<uint32_t const*>(&l);
    }
    int const off = aOff(r, c0, kP);
    uint4* p = reinterpret_cast<uint4*>(hi + off);
    p[0] = make_uint4(wh[0], wh[1], wh[2], wh[3]);
    p[8] = make_uint4(wh[4], wh[5], wh[6], wh[7]);   // next core matrix: +128 B
    if (lo)
    {
        uint4* q = reinterpret_cast<uint4*>(lo + off);
        q[0] = make_uint4(wl[0], wl[1], wl[2], wl[3]);
        q[8] = make_uint4(wl[4], wl[5], wl[6], wl[7]);
    }
}

// Activation value and derivative in FP32 (NeuralNetwork::propagateLayer).
__device__ __forceinline__ void actF(int a, float x, float& v, float& dv)
{
    switch (a)
    {
    case 0: v = x; dv = 1.0f; return;
    case 1:
    {
        float const t = tanhf(x);
        v = t;
        dv = 1.0f - t * t;
        return;
    }
    case 2:
        if (x > kExpLimitF) { v = 1.0f; dv = 0.0f; return; }
        if (x < -kExpLimitF) { v = 0.0f; dv = 0.0f; return; }
        {
            float const t = 1.0f / (1.0f + expf(-x));
            v = t;
            dv = t * (1.0f - t);
        }
        return;
    case 3:
        if (x > kExpLimitF) { v = x; dv = 1.0f; return; }
        if (x < -kExpLimitF) { v = 0.0f; dv = 0.0f; return; }
        {
            float const t = expf(x);
            v = log1pf(t);
            dv = 1.0f / (1.0f + 1.0f / t);
        }
        return;
    case 4:
        if (x > 0.0f) { v = x; dv = 1.0f; }
        else { v = 0.0f; dv = 0.0f; }
        return;
    case 5:
    {
        float const t = expf(-0.5f * x * x);
        v = t;
        dv = -x * t;
        return;
    }
    case 6: v = cosf(x); dv = -sinf(x); return;
    case 7:
    {
        float const t = 1.0f / (1.0f + expf(-x));
        v = 1.0f - t;
        dv = t * (t - 1.0f);
        return;
    }
    case 8:
    {
        float const t = expf(-x);
        v = t;
        dv = -t;
        return;
    }
    default: v = x * x; dv = 2.0f * x; return;
    }
}

// One GEMM D[128 x nP] = A[128 x kP] B[nP x kP]^T into tensor memory:
// split 0: D = Ah Bh; 1 (weights split): D = Ah Bh + Ah Bl; 2 (both
// split): D = Ah Bh + Ah Bl + Al Bh.  All threads call it after writing
// their operand rows; returns false (for every thread) when the completion
// wait gave up.
__device__ __forceinline__ bool tcGemm(uint32_t tmemD, uint32_t aH,
                                       uint32_t aL, uint32_t bH, uint32_t bL,
                                       int kP, int nP, int split, uint32_t bar,
                                       uint32_t& phase, int volatile* sAbort)
{
    proxyFence();
    tcFenceBefore();
    __syncthreads();
    if (threadIdx.x == 0)
    {
        tcFenceAfter();
        uint32_t const id = idescBF16(nP);
        uint32_t const sbo = (uint32_t)kP * 16u;
        for (int s = 0; s < kP / 16; ++s)
        {
            uint32_t const o = (uint32_t)s * 256u;
            uint64_t const ah = ummaDesc(aH + o, 128, sbo);
            uint64_t const bh = ummaDesc(bH + o, 128, sbo);
            mmaBF16(tmemD, ah, bh, id, s > 0 ? 1u : 0u);
            if (split >= 1)
                mmaBF16(tmemD, ah, ummaDesc(bL + o, 128, sbo), id, 1u);
            if (split >= 2)
                mmaBF16(tmemD, ummaDesc(aL + o, 128, sbo), bh, id, 1u);
        }
        mmaCommit(bar);
    }
    bool const ok = barWait(bar, phase);
    phase ^= 1u;
    if (!ok) *sAbort = 1;
    __syncthreads();
    if (*sAbort) return false;
    tcFenceAfter();
    return true;
}

__global__ void __launch_bounds__(kTcThreads, 1)
nnTcKernel(__grid_constant__ TcNNParams const P,
           __grid_constant__ TcNNLaunch const L)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    TcSmemLayout const lay = tcLayout(P);
    unsigned char* const sW = sm;
    float* const sF = reinterpret_cast<float*>(sm + lay.offF);
    unsigned char* const sAh = sm + lay.offAh;
    unsigned char* const sAl = P.split ? sm + lay.offAl : nullptr;
    uint64_t* const sBar = reinterpret_cast<uint64_t*>(sm + lay.offBar);
    uint32_t* const sTmem = reinterpret_cast<uint32_t*>(sm + lay.offBar + 8);
    int volatile* const sAbort =
        reinterpret_cast<int volatile*>(sm + lay.offBar + 12);
    int const tid = threadIdx.x;
    int const warp = tid >> 5;
    int const lane = tid & 31;
    if (L.status[ST_FLAGS] & FLAG_ABORT) return;
    // Tiles of 128 atoms per element (uniform over the CTA).
    int tileBeg[kMaxElem + 1];
    int count[kMaxElem];
    tileBeg[0] = 0;
    for (int e = 0; e < P.numElements; ++e)
    {
        count[e] = L.listCount ? L.listCount[e]
                               : L.es.start[e + 1] - L.es.start[e];
        tileBeg[e + 1] = tileBeg[e] + (count[e] + kTcRows - 1) / kTcRows;
    }
    int const total = tileBeg[P.numElements];
    if ((int)blockIdx.x >= total) return;

    uint32_t const bar = smemAddr(sBar);
    if (tid == 0)
    {
        barInit(bar, 1);
        *sAbort = 0;
    }
    if (warp == 0)
    {
        asm volatile(
            "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
            :: "r"(smemAddr(sTmem)), "r"((uint32_t)P.tmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;"
                     ::: "memory");
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    uint32_t const tmem = *sTmem;
    uint32_t const tRow = tmem + ((uint32_t)(warp * 32) << 16);
    uint32_t const aH = smemAddr(sAh);
    uint32_t const aL = P.split ? smemAddr(sAl) : aH;
    uint32_t phase = 0;
    int loaded = -1;
    bool ok = true;
    int const r = tid;

    for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x)
    {
        int e = 0;
        while (tile >= tileBeg[e + 1]) ++e;
        TcNet const& N = P.net[e];
        if (e != loaded)
        {
            __syncthreads();
            uint4 const* src = reinterpret_cast<uint4 const*>(L.wblob + N.wOff);
            uint4* dst = reinterpret_cast<uint4*>(sW);
            for (int k = tid; k < N.wBytes / 16; k += kTcThreads)
                dst[k] = src[k];
            for (int k = tid; k < N.fCount; k += kTcThreads)
                sF[k] = L.fblob[N.fOff + k];
            loaded = e;
            __syncthreads();
        }
        uint32_t const w0 = smemAddr(sW);
        int const row0 = L.es.start[e] + (tile - tileBeg[e]) * kTcRows;
        int const rowEnd = L.es.start[e] + count[e];
        bool const valid = row0 + r < rowEnd;
        int const atom = valid ? L.atomsByElem[row0 + r] : -1;

        // Input tile: scaled symmetry functions as BF16 (warp w loads rows
        // 32w .. 32w + 31, lanes over columns).
        for (int rr = 0; rr < 32; ++rr)
        {
            int const row = warp * 32 + rr;
            int const at = (row0 + row < rowEnd) ? L.atomsByElem[row0 + row]
                                                 : -1;
            for (int k = lane; k < N.ninP; k += 32)
            {
                float v = 0.0f;
                if (at >= 0 && k < N.nin) v = L.G[(long)at * L.maxSF + k];
                __nv_bfloat16 const h = __float2bfloat16_rn(v);
                int const off = aOff(row, k, N.ninP);
                *reinterpret_cast<__nv_bfloat16*>(sAh + off) = h;
                if (N.layer[0].splitF == 2)
                    *reinterpret_cast<__nv_bfloat16*>(sAl + off) =
                        __float2bfloat16_rn(v - __bfloat162float(h));
            }
        }

        // Forward sweep.
        float eAcc = 0.0f;
        for (int l = 0; l < N.hidden && ok; ++l)
        {
            TcLayer const& Ly = N.layer[l];
            ok = tcGemm(tmem, aH, aL, w0 + Ly.w, w0 + Ly.wl, Ly.inP, Ly.outP,
                        Ly.splitF, bar, phase, sAbort);
            if (!ok) break;
            float const* b = sF + Ly.b;
            bool const last = (l == N.hidden - 1);
            for (int c0 = 0; c0 < Ly.outP; c0 += 16)
            {
                float v[16], d[16];
                tmemLd16(tRow + c0, v);
#pragma unroll
                for (int q = 0; q < 16; ++q)
                {
                    float a, da;
                    actF(Ly.act, v[q] + b[c0 + q], a, da);
                    v[q] = a;
                    d[q] = da;
                }
                tmemSt16(tRow + Ly.fp + c0, d);
                if (!last)
                    store16(sAh, N.layer[l + 1].splitF == 2 ? sAl : nullptr,
                            r, c0, Ly.outP, v);
                else
                {
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        eAcc += sF[N.outW + c0 + q] * v[q];
                }
            }
            tmemWaitSt();
        }
        if (!ok) break;
        float E, dEz;
        actF(N.outAct, eAcc + sF[N.outB], E, dEz);
        if (valid) L.energy[atom] = (double)E;
        if (!L.derivatives) continue;

        // Backward sweep.
        {
            TcLayer const& LH = N.layer[N.hidden - 1];
            for (int c0 = 0; c0 < LH.outP; c0 += 16)
            {
                float v[16];
                tmemLd16(tRow + LH.fp + c0, v);
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    v[q] *= dEz * sF[N.outW + c0 + q];
                store16(sAh, LH.splitB == 2 ? sAl : nullptr, r, c0, LH.outP,
                        v);
            }
        }
        for (int l = N.hidden - 1; l >= 0 && ok; --l)
        {
            TcLayer const& Ly = N.layer[l];
            ok = tcGemm(tmem, aH, aL, w0 + Ly.wt, w0 + Ly.wtl, Ly.outP,
                        Ly.inP, Ly.splitB, bar, phase, sAbort);
            if (!ok) break;
            if (l > 0)
            {
                TcLayer const& Lp = N.layer[l - 1];
                for (int c0 = 0; c0 < Ly.inP; c0 += 16)
                {
                    float v[16], d[16];
                    tmemLd16(tRow + c0, v);
                    tmemLd16(tRow + Lp.fp + c0, d);
#pragma unroll
                    for (int q = 0; q < 16; ++q) v[q] *= d[q];
                    store16(sAh, Lp.splitB == 2 ? sAl : nullptr, r, c0,
                            Ly.inP, v);
                }
            }
            else
            {
                float* o = L.dEdG + (long)(valid ? atom : 0) * L.maxSF;
                for (int c0 = 0; c0 < Ly.inP; c0 += 16)
                {
                    float v[16];
                    tmemLd16(tRow + c0, v);
                    if (valid)
                    {
#pragma unroll
                        for (int q = 0; q < 16; ++q)
                            if (c0 + q < N.nin) o[c0 + q] = v[q];
                    }
                }
            }
        }
    }

    // Clean-up: after a timeout, wait (bounded) for the MMAs still in flight
    // before releasing their tensor memory.
    if (!ok && tid == 0)
    {
        atomicOr(&L.status[ST_FLAGS], FLAG_TC_TIMEOUT);
        barWait(bar, phase ^ 1u);
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if (warp == 0)
    {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"((uint32_t)P.tmemCols) : "memory");
    }
}

} // namespace

// Host: tensor-core tables and blobs from the FP64 weight blob (W out x in
// row-major at woff, bias at boff; NeuralNetwork::setConnections order
// already resolved).  normalize_nodes (division of a neuron's input sum by
// the previous layer's width) is folded into W and b.
namespace
{

uint16_t bf16Bits(float f)
{
    // Round to nearest even, as __float2bfloat16_rn (finite inputs).
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

float bf16Value(uint16_t h)
{
    uint32_t const u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// One K-major UMMA tile (rows x cols, padded rP x cP) of the high or low
// BF16 parts of value(r, c).
template <typename F>
std::vector<unsigned char> ummaTile(int rows, int cols, int rP, int cP,
                                    bool low, F value)
{
    std::vector<unsigned char> t((std::size_t)rP * cP * 2, 0);
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c)
        {
            float const x = (float)value(r, c);
            uint16_t h = bf16Bits(x);
            if (low) h = bf16Bits(x - bf16Value(h));
            std::memcpy(&t[aOff(r, c, cP)], &h, 2);
        }
    return t;
}

} // namespace

bool tcBuild(NNParams const& nn, std::vector<double> const& blob, int split,
             TcNNParams& P, std::vector<unsigned char>& wblob,
             std::vector<float>& fblob, std::string& why)
{
    std::memset(&P, 0, sizeof(P));
    wblob.clear();
    fblob.clear();
    P.numElements = nn.numElements;
    P.split = split ? 1 : 0;   // some activations split: the low tile
    auto pad16 = [](int x) { return (x + 15) / 16 * 16; };
    int maxP = 16, wMax = 0, fMax = 0, accCols = 16, fpCols = 0;
    for (int e = 0; e < nn.numElements; ++e)
    {
        TcNet& N = P.net[e];
        int const L = nn.numLayers[e];
        if (L < 3)
        {
            why = "the tensor-core form needs at least one hidden layer";
            return false;
        }
        if (nn.width[e][L - 1] != 1)
        {
            why = "the tensor-core form needs a single output neuron";
            return false;
        }
        N.hidden = L - 2;
        N.nin = nn.width[e][0];
        N.ninP = pad16(N.nin);
        N.wOff = (long)wblob.size();
        N.fOff = (long)fblob.size();
        std::vector<unsigned char> region;
        std::vector<float> freg;
        int fp = 0;
        auto append = [&](std::vector<unsigned char> const& t) {
            int const at = (int)region.size();
            region.insert(region.end(), t.begin(), t.end());
            return at;
        };
        for (int h = 0; h < N.hidden; ++h)
        {
            int const l = h + 1;     // layer index in NNParams
            TcLayer& Ly = N.layer[h];
            Ly.in = nn.width[e][l - 1];
            Ly.out = nn.width[e][l];
            Ly.inP = pad16(Ly.in);
            Ly.outP = pad16(Ly.out);
            Ly.act = nn.act[e][l];
            if (Ly.inP > 256 || Ly.outP > 256)
            {
                why = "a layer is wider than 256 neurons";
                return false;
            }
            maxP = std::max(maxP, std::max(Ly.inP, Ly.outP));
            accCols = std::max(accCols, std::max(Ly.inP, Ly.outP));
            double const norm = nn.normalizeNeurons ? 1.0 / Ly.in : 1.0;
            double const* W = blob.data() + nn.woff[e][l];
            double const* b = blob.data() + nn.boff[e][l];
            int const ni = Ly.in;
            auto w = [&](int o, int j) { return W[(long)o * ni + j] * norm; };
            auto wt = [&](int j, int o) { return W[(long)o * ni + j] * norm; };
            // Per GEMM: 2 = activations and weights split, 1 = weights only.
            Ly.splitF = split ? 2 : 0;
            Ly.splitB = (split == 1 || (split == 2 && h == 0)) ? 2
                      : (split == 2) ? 1 : 0;
            Ly.w = append(ummaTile(Ly.out, Ly.in, Ly.outP, Ly.inP, false, w));
            Ly.wl = Ly.splitF ? append(ummaTile(Ly.out, Ly.in, Ly.outP,
                                                Ly.inP, true, w))
                              : Ly.w;
            Ly.wt = append(ummaTile(Ly.in, Ly.out, Ly.inP, Ly.outP, false, wt));
            Ly.wtl = Ly.splitB ? append(ummaTile(Ly.in, Ly.out, Ly.inP,
                                                 Ly.outP, true, wt))
                               : Ly.wt;
            Ly.b = (int)freg.size();
            for (int o = 0; o < Ly.outP; ++o)
                freg.push_back(o < Ly.out ? (float)(b[o] * norm) : 0.0f);
            Ly.fp = fp;              // relative; made absolute below
            fp += Ly.outP;
        }
        fpCols = std::max(fpCols, fp);
        // Output neuron.
        {
            int const l = L - 1;
            int const ni = nn.width[e][l - 1];
            int const niP = pad16(ni);
            double const norm = nn.normalizeNeurons ? 1.0 / ni : 1.0;
            double const* W = blob.data() + nn.woff[e][l];
            double const* b = blob.data() + nn.boff[e][l];
            N.outAct = nn.act[e][l];
            N.outW = (int)freg.size();
            for (int j = 0; j < niP; ++j)
                freg.push_back(j < ni ? (float)(W[j] * norm) : 0.0f);
            N.outB = (int)freg.size();
            freg.push_back((float)(b[0] * norm));
        }
        N.wBytes = (int)region.size();
        N.fCount = (int)freg.size();
        wblob.insert(wblob.end(), region.begin(), region.end());
        fblob.insert(fblob.end(), freg.begin(), freg.end());
        while (fblob.size() % 4) fblob.push_back(0.0f);
        wMax = std::max(wMax, N.wBytes);
        fMax = std::max(fMax, N.fCount);
    }
    // Tensor memory: accumulators in [0, accCols), then the f' columns.
    for (int e = 0; e < nn.numElements; ++e)
        for (int h = 0; h < P.net[e].hidden; ++h)
            P.net[e].layer[h].fp += accCols;
    int cols = 32;
    while (cols < accCols + fpCols) cols <<= 1;
    if (cols > 512)
    {
        why = "the hidden layers need more than 512 tensor-memory columns";
        return false;
    }
    P.tmemCols = cols;
    P.maxP = maxP;
    P.wMax = (wMax + 127) / 128 * 128;
    P.fMax = fMax;
    P.smemBytes = tcLayout(P).total;
    if (P.smemBytes > 227 * 1024)
    {
        why = "the network needs " + std::to_string(P.smemBytes)
            + " bytes of shared memory per tile (at most 232448)";
        return false;
    }
    return true;
}

void launchNeuralNetworksTC(TcNNParams const& P, TcNNLaunch const& L,
                            cudaStream_t s)
{
    cudaFuncSetAttribute(nnTcKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         P.smemBytes);
    // Upper bound of the tile count (all atoms); CTAs beyond the actual
    // count return before allocating tensor memory.
    int total = 0;
    for (int e = 0; e < P.numElements; ++e)
        total += (L.es.start[e + 1] - L.es.start[e] + kTcRows - 1) / kTcRows;
    int const grid = std::max(1, std::min(total, L.grid));
    noteLaunches(1);
    nnTcKernel<<<grid, kTcThreads, P.smemBytes, s>>>(P, L);
}

int tcBlocksPerSM(TcNNParams const& P)
{
    cudaFuncSetAttribute(nnTcKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         P.smemBytes);
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &blocks, nnTcKernel, kTcThreads, P.smemBytes) != cudaSuccess
        || blocks < 1)
        blocks = 1;
    // Tensor memory: 512 columns per SM shared by the resident CTAs.
    return std::max(1, std::min(blocks, 512 / P.tmemCols));
}

} // namespace n2p2b
