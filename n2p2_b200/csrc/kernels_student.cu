// Training of the distilled student network: per-atom energy and force
// matching against a teacher, with hand-written Adam.
//
// Student per element: one hidden layer, E = w2 . tanh(W1 G + b1) + b2
// (input -> H -> 1), evaluated in FP32 on the symmetry functions G that the
// teacher's potential defines.  One optimizer step over a batch B of atoms:
//
//   loss = wE / |B| sum_{i in B} (E_i - E_i^T)^2
//        + wF / (3|B|) sum_{i in B} |F_i - F_i^T|^2,
//   F_i  = -sum_j sum_s (dE_j/dG_js) dG_js/dr_i          (Mode::calculateForces)
//
// The force term's gradient needs, for every atom j near the batch, the
// adjoint u_js = -2 wF / (3|B|) sum_{i in B} r_i . dG_js/dr_i (r_i the force
// residual; with dG_j/dr_j = -sum over j's entries of the neighbor slots,
// u_js = -2 wF / (3|B|) sum_e (r_i(e) - r_j) . slot_e, r_i(e) = 0 for
// entries that are images of j itself), after which
//   d loss / d theta = sum_j [ c_j dE_j/d theta + d (u_j . dE_j/dG_j) / d theta ],
//   c_j = 2 wE / |B| (E_j - E_j^T) for j in B, else 0.
// With h = tanh(z), t = 1 - h^2 and a = W1 u_j the second term is
//   d/dw2_k = a_k t_k,  d/dW1_kl = u_l w2_k t_k - 2 a_k w2_k h_k t_k G_l,
//   d/db1_k = -2 a_k w2_k h_k t_k,
// so per atom the W1 gradient is alpha_k G_l + beta_k u_l with
//   alpha_k = w2_k t_k (c_j - 2 a_k h_k),  beta_k = w2_k t_k.
//
// Kernels: residuals of the batch atoms; the adjoint (warp per atom j over
// its neighbor entries, the layout of the force kernel); per-block partial
// gradients (64 atoms of one element per block); a fixed-order reduction of
// the partials fused with the Adam update (Kingma & Ba, bias-corrected; the
// W1 learning rate is divided per input by that symmetry function's sigma,
// i.e. Adam on the weights of standardized inputs G / sigma); and
// the training range of the symmetry functions (per-SF min / max of the
// unscaled values) that gates the student at inference.
#include <cfloat>

#include "device_common.cuh"
#include "kernels.h"

namespace n2p2b
{

namespace
{

constexpr int kGradRows = 64;
constexpr int kGradThreads = 128;

__global__ void residualKernel(StudentLaunch const L)
{
    int const b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= L.batchSize) return;
    int const i = L.batch[b];
    double const rE = L.Ei[i] * L.eScale - L.labelE[i];
    double r2 = 0.0;
    L.rE[i] = (float)rE;
    for (int c = 0; c < 3; ++c)
    {
        double const r = L.F[(long)i * 3 + c] - L.labelF[(long)i * 3 + c];
        L.rF[(long)i * 3 + c] = (float)r;
        r2 += r * r;
    }
    atomicAdd(&L.loss[0], rE * rE);
    atomicAdd(&L.loss[1], r2);
}

// Warp per atom j: u_j over its symmetry functions.
template <typename T>
__global__ void __launch_bounds__(128)
adjointKernel(StudentLaunch const L)
{
    extern __shared__ float usm[];
    int const lane = threadIdx.x & 31;
    int const w = threadIdx.x >> 5;
    int const warps = blockDim.x >> 5;
    float* acc = usm + (long)w * L.maxSF;
    T const* const nbr = static_cast<T const*>(L.dGdr);
    float const scale = (float)(-2.0 * L.wF * L.fScale
                                / (3.0 * L.batchSize));
    for (int j = blockIdx.x * warps + w; j < L.n; j += gridDim.x * warps)
    {
        int const ej = L.elem[j];
        int const nsf = L.numSF[ej];
        float const rx = L.rF[(long)j * 3 + 0];
        float const ry = L.rF[(long)j * 3 + 1];
        float const rz = L.rF[(long)j * 3 + 2];
        for (int s = lane; s < nsf; s += 32) acc[s] = 0.0f;
        __syncwarp();
        long const b = L.nbrOff[j];
        int const cnt = L.nbrOff[j + 1] - (int)b;
        T const* gd = nbr + b * (long)L.maxSlots * 3;
        int seg = 0;
        for (int en = 0; en < L.numElements; ++en)
        {
            int const sb = seg;
            int const se = seg + L.nbrCountElem[(long)j * L.numElements + en];
            seg = se;
            int const ns = L.numSlots[ej][en];
            int16_t const* tab = L.slotSF + ((long)ej * kMaxElem + en)
                                            * L.maxSlots;
            for (int sl = 0; sl < ns; ++sl)
            {
                float v = 0.0f;
                for (int t = sb + lane; t < se; t += 32)
                {
                    int const i = L.nbrIdx[b + t];
                    // A periodic self image carries no pair force, only its
                    // share of j's self derivative.
                    float qx = -rx, qy = -ry, qz = -rz;
                    if (i != j)
                    {
                        qx += L.rF[(long)i * 3 + 0];
                        qy += L.rF[(long)i * 3 + 1];
                        qz += L.rF[(long)i * 3 + 2];
                    }
                    v += qx * (float)gd[((long)sl * 3 + 0) * cnt + t]
                       + qy * (float)gd[((long)sl * 3 + 1) * cnt + t]
                       + qz * (float)gd[((long)sl * 3 + 2) * cnt + t];
                }
                v = warpSumF(v);
                if (lane == 0) acc[tab[sl]] += v;
                __syncwarp();
            }
        }
        for (int s = lane; s < nsf; s += 32)
            L.u[(long)j * L.maxSF + s] = scale * acc[s];
        __syncwarp();
    }
}

// Partial gradients of 64 atoms of one element per block.
template <typename T>
__global__ void __launch_bounds__(kGradThreads)
gradKernel(StudentLaunch const L)
{
    extern __shared__ float gsm[];
    int e = 0;
    while ((int)blockIdx.x >= L.blkBeg[e + 1]) ++e;
    int const nin = L.numSF[e];
    int const H = L.hidden[e];
    int const row0 = L.es.start[e] + ((int)blockIdx.x - L.blkBeg[e]) * kGradRows;
    int const rows = min(kGradRows, L.es.start[e + 1] - row0);
    int const ld = nin + 1;
    float* sG = gsm;                          // [rows][nin + 1]
    float* sU = sG + kGradRows * ld;          // [rows][nin + 1]
    float* sA = sU + kGradRows * ld;          // alpha [rows][H]
    float* sB = sA + kGradRows * H;           // beta
    float* sC = sB + kGradRows * H;           // gamma (w2 gradient)
    float* sc = sC + kGradRows * H;           // c per row
    float* sW = sc + kGradRows;               // W1 [H][ldw]
    int const ldw = nin | 1;                  // odd stride: no bank conflicts
    T const* const G = static_cast<T const*>(L.G);
    float const* const wb = L.blob;
    float const* W1 = wb + L.woff1[e];
    float const* b1 = wb + L.boff1[e];
    float const* w2 = wb + L.woff2[e];
    for (int q = threadIdx.x; q < H * nin; q += blockDim.x)
        sW[(q / nin) * ldw + q % nin] = W1[q];
    int const lane = threadIdx.x & 31;
    int const warp = threadIdx.x >> 5;
    for (int r = warp; r < kGradRows; r += blockDim.x >> 5)
    {
        int const atom = r < rows ? L.atomsByElem[row0 + r] : -1;
        for (int l = lane; l < nin; l += 32)
        {
            sG[r * ld + l] = atom >= 0 ? (float)G[(long)atom * L.maxSF + l]
                                       : 0.0f;
            sU[r * ld + l] = atom >= 0 ? L.u[(long)atom * L.maxSF + l] : 0.0f;
        }
    }
    __syncthreads();
    float const cE = (float)(2.0 * L.wE * L.eScale / L.batchSize);
    // Thread per (row, neuron): z = W1 G + b1 and a = W1 u.
    for (int q = threadIdx.x; q < kGradRows * H; q += blockDim.x)
    {
        int const r = q / H, k = q - (q / H) * H;
        int const atom = r < rows ? L.atomsByElem[row0 + r] : -1;
        float const c = atom >= 0 ? cE * L.rE[atom] : 0.0f;
        if (k == 0) sc[r] = c;
        float z = b1[k], a = 0.0f;
        for (int l = 0; l < nin; ++l)
        {
            z += sW[k * ldw + l] * sG[r * ld + l];
            a += sW[k * ldw + l] * sU[r * ld + l];
        }
        float const h = tanhf(z);
        float const t = 1.0f - h * h;
        bool const live = atom >= 0;
        sA[r * H + k] = live ? w2[k] * t * (c - 2.0f * a * h) : 0.0f;
        sB[r * H + k] = live ? w2[k] * t : 0.0f;
        sC[r * H + k] = live ? c * h + a * t : 0.0f;
    }
    __syncthreads();
    float* out = L.gpart + (long)blockIdx.x * L.paramStride;
    int const nW = H * nin;
    int const np = nW + 2 * H + 1;
    for (int p = threadIdx.x; p < np; p += blockDim.x)
    {
        float g = 0.0f;
        if (p < nW)
        {
            int const k = p / nin, l = p - (p / nin) * nin;
            for (int r = 0; r < kGradRows; ++r)
                g += sA[r * H + k] * sG[r * ld + l]
                   + sB[r * H + k] * sU[r * ld + l];
        }
        else if (p < nW + H)
        {
            int const k = p - nW;
            for (int r = 0; r < kGradRows; ++r) g += sA[r * H + k];
        }
        else if (p < nW + 2 * H)
        {
            int const k = p - nW - H;
            for (int r = 0; r < kGradRows; ++r) g += sC[r * H + k];
        }
        else
        {
            for (int r = 0; r < kGradRows; ++r) g += sc[r];
        }
        out[p] = g;
    }
}

// Sum of the partials (fixed order) + Adam, thread per parameter.
__global__ void adamKernel(StudentLaunch const L)
{
    int const e = blockIdx.y;
    int const nin = L.numSF[e];
    int const H = L.hidden[e];
    int const nW = H * nin;
    int const np = nW + 2 * H + 1;
    int const p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    float g = 0.0f;
    for (int b = L.blkBeg[e]; b < L.blkBeg[e + 1]; ++b)
        g += L.gpart[(long)b * L.paramStride + p];
    long pos, posT = -1;
    float lr = L.lr;
    if (p < nW)
    {
        int const k = p / nin, l = p - (p / nin) * nin;
        pos = L.woff1[e] + p;
        posT = L.wtoff1[e] + (long)l * H + k;
        if (L.lrScale) lr *= L.lrScale[(long)e * L.maxSF + l];
    }
    else if (p < nW + H) pos = L.boff1[e] + (p - nW);
    else if (p < nW + 2 * H)
    {
        pos = L.woff2[e] + (p - nW - H);
        posT = L.wtoff2[e] + (p - nW - H);
    }
    else pos = L.boff2[e];
    if (L.grad) L.grad[pos] = g;
    float const m = L.beta1 * L.m[pos] + (1.0f - L.beta1) * g;
    float const v = L.beta2 * L.v[pos] + (1.0f - L.beta2) * g * g;
    L.m[pos] = m;
    L.v[pos] = v;
    float const mh = m / L.bc1;
    float const vh = v / L.bc2;
    float const w = L.blob[pos] - lr * mh / (sqrtf(vh) + L.epsAdam);
    L.blob[pos] = w;
    if (posT >= 0) L.blob[posT] = w;
}

__device__ __forceinline__ void atomicMinD(double* a, double v)
{
    unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
    unsigned long long old = *p;
    while (v < __longlong_as_double((long long)old))
    {
        unsigned long long const prev =
            atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
        if (prev == old) break;
        old = prev;
    }
}

__device__ __forceinline__ void atomicMaxD(double* a, double v)
{
    unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
    unsigned long long old = *p;
    while (v > __longlong_as_double((long long)old))
    {
        unsigned long long const prev =
            atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
        if (prev == old) break;
        old = prev;
    }
}

// Training range: per (element, SF) min / max of the unscaled values over
// 256-atom chunks of each element, one atomic per chunk and SF.
template <typename T>
__global__ void rangeKernel(RangeLaunch const L)
{
    int e = 0;
    while ((int)blockIdx.x >= L.blkBeg[e + 1]) ++e;
    int const r0 = L.es.start[e] + ((int)blockIdx.x - L.blkBeg[e]) * 256;
    int const r1 = min(r0 + 256, L.es.start[e + 1]);
    T const* const G = static_cast<T const*>(L.G);
    for (int s = threadIdx.x; s < L.numSF[e]; s += blockDim.x)
    {
        SFScale const q = L.scale[(long)e * L.maxSF + s];
        double lo = DBL_MAX, hi = -DBL_MAX;
        for (int r = r0; r < r1; ++r)
        {
            int const a = L.atomsByElem[r];
            double const g = (double)G[(long)a * L.maxSF + s];
            double const v = (g - q.smin) / q.b + q.shift;
            lo = fmin(lo, v);
            hi = fmax(hi, v);
        }
        atomicMinD(&L.range[(long)e * L.maxSF + s].lo, lo);
        atomicMaxD(&L.range[(long)e * L.maxSF + s].hi, hi);
    }
}

} // namespace

std::size_t studentGradSmem(int maxNin, int maxH)
{
    return sizeof(float) * ((std::size_t)2 * kGradRows * (maxNin + 1)
                            + (std::size_t)3 * kGradRows * maxH + kGradRows
                            + (std::size_t)maxH * (maxNin | 1));
}

int studentGradBlocks(ElemStarts const& es, int numElements, int* blkBeg)
{
    blkBeg[0] = 0;
    for (int e = 0; e < numElements; ++e)
        blkBeg[e + 1] = blkBeg[e]
                      + (es.start[e + 1] - es.start[e] + kGradRows - 1)
                        / kGradRows;
    for (int e = numElements + 1; e <= kMaxElem; ++e)
        blkBeg[e] = blkBeg[numElements];
    return blkBeg[numElements];
}

void launchStudentTrainStep(StudentLaunch const& L, std::size_t gradSmem,
                            int maxParams, cudaStream_t s)
{
    bool const f = L.precision != PREC_FP64;
    noteLaunches(4);
    residualKernel<<<(L.batchSize + 127) / 128 > 0
                         ? (L.batchSize + 127) / 128 : 1, 128, 0, s>>>(L);
    int const warps = 4;
    std::size_t const ush = sizeof(float) * warps * (std::size_t)L.maxSF;
    int const ag = (L.n + warps - 1) / warps;
    if (f) adjointKernel<float><<<ag, 32 * warps, ush, s>>>(L);
    else adjointKernel<double><<<ag, 32 * warps, ush, s>>>(L);
    int const blocks = L.blkBeg[L.numElements];
    if (f)
    {
        cudaFuncSetAttribute(gradKernel<float>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gradSmem);
        gradKernel<float><<<blocks, kGradThreads, gradSmem, s>>>(L);
    }
    else
    {
        cudaFuncSetAttribute(gradKernel<double>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gradSmem);
        gradKernel<double><<<blocks, kGradThreads, gradSmem, s>>>(L);
    }
    dim3 const ag2((maxParams + 255) / 256, L.numElements);
    adamKernel<<<ag2, 256, 0, s>>>(L);
}

void launchStudentRange(RangeLaunch const& L, cudaStream_t s)
{
    noteLaunches(1);
    int const blocks = L.blkBeg[L.numElements];
    if (blocks <= 0) return;
    if (L.precision != PREC_FP64)
        rangeKernel<float><<<blocks, 128, 0, s>>>(L);
    else
        rangeKernel<double><<<blocks, 128, 0, s>>>(L);
}

} // namespace n2p2b
