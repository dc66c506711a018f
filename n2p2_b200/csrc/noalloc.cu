// n2p2b_neighbor_list_noalloc: a neighbor list (the reference's
// Structure::calculateNeighborList semantics: every (j, image) with
// |r_i - r_j + image|^2 <= rc^2, in (j ascending, image) order) that
// allocates no memory.
//
// Who needs it: callers that must not allocate device memory at run time --
// e.g. an MD engine that reserves all GPU memory up front and hands out
// fixed buffers, or a host that drives the GPU from a context where
// cudaMalloc/cudaFree would synchronize the device or is forbidden (signal
// handlers, real-time loops, code running between a caller's own
// allocations).  The caller owns every input and output buffer; the only
// other memory used is the scratch below.
//
// Scratch: one file-scope __device__ array of kScratchInts ints (about
// 1.3 MB), held by every GPU that loads this library until process exit.
// It bounds the problem size: at most kMaxAtoms atoms, kMaxCells cell bins
// and kMaxNeighbors neighbors per atom; larger inputs are rejected before
// any launch.  Every call reuses the same array and leaves its last contents
// there; the parts that must start at zero are cleared at the start of each
// call.  Two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on the scratch and corrupt each other's
// results: serialize them.
//
// In host code the array's name is only a host-side stand-in; its device
// address is obtained once per device with cudaGetSymbolAddress (with that
// device current) on the first call made for the device, so that first call
// should come before any stream capture.  Under CUDA's lazy module loading
// (the default) that first call is also when the library's device code and
// this array are loaded onto the device, which takes device memory: make
// one warm-up call before the host reserves its memory (or set
// CUDA_MODULE_LOADING=EAGER).  Every call waits on the host until its
// stream has finished the work (it reads the status words back).
#include "n2p2_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace
{

constexpr long kMaxAtoms = 65536;
constexpr long kMaxCells = 65536;
constexpr int kMaxNeighbors = 1024;
constexpr int kStatusInts = 16;
// cellOf + cellAtoms (atoms), cellCount + cellFill + cellStart (cells + 1),
// status words.
constexpr long kScratchInts = 2 * kMaxAtoms + 3 * (kMaxCells + 1)
                            + kStatusInts;

static __device__ __align__(256) int g_scratch[kScratchInts];

constexpr int kWarpsPerBlock = 4;
constexpr unsigned kFull = 0xffffffffu;

enum
{
    S_FLAGS = 0,
    S_TOTAL_LO = 1,   // total entries, low and high 32 bits (unclamped)
    S_TOTAL_HI = 2,
    S_MAXNBR = 3
};
enum
{
    F_OUTSIDE = 1,
    F_OVERFLOW = 2,
    F_TOO_MANY_NEIGHBORS = 4
};

struct Geo
{
    int    periodic;
    int    pbc[3];
    int    ncell[3];
    int    nimg;
    double box[3][3];
    double invbox[3][3];
    double rc2;
};

struct Scratch
{
    int* cellOf;
    int* cellAtoms;
    int* cellCount;
    int* cellFill;
    int* cellStart;
    int* status;
};

// --- exact reference displacement (no contraction, Vec3D association) ----
__device__ __forceinline__ bool pairTest(Geo const& g, double const ri[3],
                                         double const* __restrict__ pos,
                                         int j, int b0, int b1, int b2,
                                         double dr[3], double& n2)
{
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        double v = __dsub_rn(ri[k], pos[3 * j + k]);
        if (g.periodic)
        {
            v = __dadd_rn(v, __dmul_rn((double)b0, g.box[0][k]));
            v = __dadd_rn(v, __dmul_rn((double)b1, g.box[1][k]));
            v = __dadd_rn(v, __dmul_rn((double)b2, g.box[2][k]));
        }
        dr[k] = v;
    }
    n2 = __dadd_rn(__dadd_rn(__dmul_rn(dr[0], dr[0]), __dmul_rn(dr[1], dr[1])),
                   __dmul_rn(dr[2], dr[2]));
    return n2 <= g.rc2;
}

__device__ __forceinline__ void decodeImage(Geo const& g, int img, int& b0,
                                            int& b1, int& b2)
{
    int const n2 = 2 * g.pbc[2] + 1;
    int const n1 = 2 * g.pbc[1] + 1;
    b2 = img % n2 - g.pbc[2];
    img /= n2;
    b1 = img % n1 - g.pbc[1];
    b0 = img / n1 - g.pbc[0];
}

__global__ void naPrepare(int n, Geo g, double const* __restrict__ pos,
                          Scratch s)
{
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c[3];
    bool inside = true;
    for (int k = 0; k < 3; ++k)
    {
        double const f = pos[3 * i] * g.invbox[0][k]
                       + pos[3 * i + 1] * g.invbox[1][k]
                       + pos[3 * i + 2] * g.invbox[2][k];
        if (!(f >= -1e-12 && f <= 1.0 + 1e-12)) inside = false;
        c[k] = min(max((int)floor(f * g.ncell[k]), 0), g.ncell[k] - 1);
    }
    if (!inside) atomicOr(&s.status[S_FLAGS], F_OUTSIDE);
    int const cell = (c[0] * g.ncell[1] + c[1]) * g.ncell[2] + c[2];
    s.cellOf[i] = cell;
    atomicAdd(&s.cellCount[cell], 1);
}

// Single-block exclusive scan of cnt[0..n) into off[0..n]; optionally checks
// the total against `capacity` and records the total / maximum.
__global__ void naScan(int n, int const* __restrict__ cnt,
                       int* __restrict__ off, long capacity,
                       int* __restrict__ status, int record)
{
    __shared__ long part[1024];
    __shared__ int mxs[1024];
    int const t = threadIdx.x;
    int const chunk = (n + blockDim.x - 1) / blockDim.x;
    int const b = min(n, t * chunk), e = min(n, b + chunk);
    long sum = 0;
    int mx = 0;
    for (int i = b; i < e; ++i)
    {
        sum += cnt[i];
        mx = max(mx, cnt[i]);
    }
    part[t] = sum;
    mxs[t] = mx;
    __syncthreads();
    if (t == 0)
    {
        long run = 0;
        int m = 0;
        for (int k = 0; k < (int)blockDim.x; ++k)
        {
            long const v = part[k];
            part[k] = run;
            run += v;
            m = max(m, mxs[k]);
        }
        off[n] = (int)min(run, (long)0x7fffffff);
        if (record)
        {
            unsigned long long const u = (unsigned long long)run;
            status[S_TOTAL_LO] = (int)(unsigned)(u & 0xffffffffull);
            status[S_TOTAL_HI] = (int)(unsigned)(u >> 32);
            status[S_MAXNBR] = m;
            // Offsets and indices are int32: a list of more than INT32_MAX
            // entries cannot be written, whatever the caller's capacity.
            if (run > capacity || run > 0x7fffffffL)
                status[S_FLAGS] |= F_OVERFLOW;
            if (m > kMaxNeighbors) status[S_FLAGS] |= F_TOO_MANY_NEIGHBORS;
        }
    }
    __syncthreads();
    long run = part[t];
    for (int i = b; i < e; ++i)
    {
        off[i] = (int)run;
        run += cnt[i];
    }
}

__global__ void naBin(int n, Scratch s)
{
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int const c = s.cellOf[i];
    s.cellAtoms[s.cellStart[c] + atomicAdd(&s.cellFill[c], 1)] = i;
}

// Cell path, warp per atom.  FILL = 0 counts; FILL = 1 collects the hits'
// keys (j * nimg + image) in shared memory, ranks them and writes the
// atom's entries in key order.
template <int FILL>
__global__ void naCell(int n, Geo g, double const* __restrict__ pos, Scratch s,
                       int* __restrict__ counts, int const* __restrict__ offsets,
                       int* __restrict__ index, double* __restrict__ dr,
                       double* __restrict__ dist)
{
    __shared__ int keys[kWarpsPerBlock][kMaxNeighbors];
    int const flags = s.status[S_FLAGS];
    if (flags & F_OUTSIDE) return;
    if (FILL && (flags & (F_OVERFLOW | F_TOO_MANY_NEIGHBORS))) return;
    int const lane = threadIdx.x & 31;
    int const w = threadIdx.x >> 5;
    int const i = blockIdx.x * kWarpsPerBlock + w;
    if (i >= n) return;
    double const ri[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    int const cell = s.cellOf[i];
    int const c[3] = {cell / (g.ncell[2] * g.ncell[1]),
                      (cell / g.ncell[2]) % g.ncell[1], cell % g.ncell[2]};
    int total = 0;
    for (int st = 0; st < 27; ++st)
    {
        int const d[3] = {st / 9 - 1, (st / 3) % 3 - 1, st % 3 - 1};
        int cc[3], bc[3];
        for (int k = 0; k < 3; ++k)
        {
            int v = c[k] + d[k], wrap = 0;
            if (v < 0) { v += g.ncell[k]; wrap = -1; }
            else if (v >= g.ncell[k]) { v -= g.ncell[k]; wrap = 1; }
            cc[k] = v;
            bc[k] = -wrap;
        }
        int const cid = (cc[0] * g.ncell[1] + cc[1]) * g.ncell[2] + cc[2];
        int const img = ((bc[0] + g.pbc[0]) * (2 * g.pbc[1] + 1)
                         + (bc[1] + g.pbc[1])) * (2 * g.pbc[2] + 1)
                      + (bc[2] + g.pbc[2]);
        bool const zero = bc[0] == 0 && bc[1] == 0 && bc[2] == 0;
        int const cs = s.cellStart[cid], cn = s.cellCount[cid];
        for (int t0 = 0; t0 < cn; t0 += 32)
        {
            int const t = t0 + lane;
            bool hit = false;
            int j = 0;
            if (t < cn)
            {
                j = s.cellAtoms[cs + t];
                if (!(j == i && zero))
                {
                    double v[3], n2;
                    hit = pairTest(g, ri, pos, j, bc[0], bc[1], bc[2], v, n2);
                }
            }
            unsigned const m = __ballot_sync(kFull, hit);
            if (FILL && hit)
            {
                int const p = total + __popc(m & ((1u << lane) - 1u));
                keys[w][p] = j * g.nimg + img;
            }
            total += __popc(m);
        }
    }
    if (!FILL)
    {
        if (lane == 0) counts[i] = total;
        return;
    }
    __syncwarp();
    long const base = offsets[i];
    for (int p = lane; p < total; p += 32)
    {
        int const k = keys[w][p];
        int r = 0;
        for (int q = 0; q < total; ++q) r += keys[w][q] < k;
        int const j = k / g.nimg;
        int b0, b1, b2;
        decodeImage(g, k % g.nimg, b0, b1, b2);
        double v[3], n2;
        pairTest(g, ri, pos, j, b0, b1, b2, v, n2);
        long const o = base + r;
        index[o] = j;
        dr[3 * o + 0] = v[0];
        dr[3 * o + 1] = v[1];
        dr[3 * o + 2] = v[2];
        dist[o] = __dsqrt_rn(n2);
    }
}

// Brute path (the reference's own enumeration order), warp per atom.
template <int FILL>
__global__ void naBrute(int n, Geo g, int onlyIfOutside,
                        double const* __restrict__ pos, Scratch s,
                        int* __restrict__ counts,
                        int const* __restrict__ offsets,
                        int* __restrict__ index, double* __restrict__ dr,
                        double* __restrict__ dist)
{
    int const flags = s.status[S_FLAGS];
    if (onlyIfOutside && !(flags & F_OUTSIDE)) return;
    if (FILL && (flags & F_OVERFLOW)) return;
    int const lane = threadIdx.x & 31;
    int const i = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    double const ri[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    long const ncand = (long)n * g.nimg;
    long const base = FILL ? (long)offsets[i] : 0;
    int total = 0;
    for (long c0 = 0; c0 < ncand; c0 += 32)
    {
        long const c = c0 + lane;
        bool hit = false;
        int j = 0;
        double v[3] = {0, 0, 0}, n2 = 0.0;
        if (c < ncand)
        {
            j = (int)(c / g.nimg);
            int b0, b1, b2;
            decodeImage(g, (int)(c % g.nimg), b0, b1, b2);
            if (!(j == i && b0 == 0 && b1 == 0 && b2 == 0))
                hit = pairTest(g, ri, pos, j, b0, b1, b2, v, n2);
        }
        unsigned const m = __ballot_sync(kFull, hit);
        if (FILL && hit)
        {
            long const o = base + total + __popc(m & ((1u << lane) - 1u));
            index[o] = j;
            dr[3 * o + 0] = v[0];
            dr[3 * o + 1] = v[1];
            dr[3 * o + 2] = v[2];
            dist[o] = __dsqrt_rn(n2);
        }
        total += __popc(m);
    }
    if (!FILL && lane == 0) counts[i] = total;
}

// --- host helpers (reference geometry, no contraction: see build flags) ---

void crossV(double const a[3], double const b[3], double w[3])
{
    w[0] = a[1] * b[2] - a[2] * b[1];
    w[1] = a[2] * b[0] - a[0] * b[2];
    w[2] = a[0] * b[1] - a[1] * b[0];
}

void normV(double v[3])
{
    double const n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= n;
    v[1] /= n;
    v[2] /= n;
}

std::mutex g_mutex;
int* g_address[64] = {};

int fail(char* err, size_t len, int code, char const* msg)
{
    if (err && len) std::snprintf(err, len, "%s", msg);
    return code;
}

} // namespace

extern "C" int n2p2b_neighbor_list_noalloc(
    int device, void* stream, int64_t num_atoms, double const* box,
    double const* positions, double cutoff, int32_t* counts, int32_t* offsets,
    int32_t* index, double* dr, double* d, int64_t capacity, int64_t* total,
    char* err, size_t err_len)
{
    if (err && err_len) err[0] = '\0';
    if (num_atoms <= 0 || !positions || !counts || !offsets || !total
        || (capacity > 0 && (!index || !dr || !d)) || !(cutoff > 0.0)
        || device < 0 || device >= 64)
        return fail(err, err_len, N2P2B_ERR_ARGUMENT,
                    "n2p2b_neighbor_list_noalloc: invalid argument");
    if (num_atoms > kMaxAtoms)
        return fail(err, err_len, N2P2B_ERR_CAPACITY,
                    "n2p2b_neighbor_list_noalloc: more atoms than its static "
                    "scratch holds (N2P2B_NOALLOC_MAX_ATOMS = 65536)");
    int const n = (int)num_atoms;

    // Geometry on the host: Structure::calculatePbcCopies and cell grid.
    Geo g;
    std::memset(&g, 0, sizeof(g));
    g.rc2 = cutoff * cutoff;
    if (box)
    {
        g.periodic = 1;
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) g.box[k][c] = box[3 * k + c];
        double const (&b)[3][3] = g.box;
        double invdet = b[0][0] * b[1][1] * b[2][2] + b[1][0] * b[2][1] * b[0][2]
                      + b[2][0] * b[0][1] * b[1][2] - b[2][0] * b[1][1] * b[0][2]
                      - b[0][0] * b[2][1] * b[1][2] - b[1][0] * b[0][1] * b[2][2];
        invdet = 1.0 / invdet;
        double (&v)[3][3] = g.invbox;
        v[0][0] = b[1][1] * b[2][2] - b[2][1] * b[1][2];
        v[0][1] = b[2][1] * b[0][2] - b[0][1] * b[2][2];
        v[0][2] = b[0][1] * b[1][2] - b[1][1] * b[0][2];
        v[1][0] = b[2][0] * b[1][2] - b[1][0] * b[2][2];
        v[1][1] = b[0][0] * b[2][2] - b[2][0] * b[0][2];
        v[1][2] = b[1][0] * b[0][2] - b[0][0] * b[1][2];
        v[2][0] = b[1][0] * b[2][1] - b[2][0] * b[1][1];
        v[2][1] = b[2][0] * b[0][1] - b[0][0] * b[2][1];
        v[2][2] = b[0][0] * b[1][1] - b[1][0] * b[0][1];
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) v[k][c] *= invdet;
        double axb[3], axc[3], bxc[3];
        crossV(b[0], b[1], axb);
        normV(axb);
        crossV(b[0], b[2], axc);
        normV(axc);
        crossV(b[1], b[2], bxc);
        normV(bxc);
        double const proj[3] = {
            std::fabs(b[0][0] * bxc[0] + b[0][1] * bxc[1] + b[0][2] * bxc[2]),
            std::fabs(b[1][0] * axc[0] + b[1][1] * axc[1] + b[1][2] * axc[2]),
            std::fabs(b[2][0] * axb[0] + b[2][1] * axb[1] + b[2][2] * axb[2])};
        long cells = 1;
        bool cellOk = true;
        for (int k = 0; k < 3; ++k)
        {
            g.pbc[k] = 0;
            while (g.pbc[k] * proj[k] <= cutoff) g.pbc[k]++;
            int nc = (int)std::floor(proj[k] / (cutoff * (1.0 + 1e-9)));
            nc = std::min(nc, 40);
            if (nc < 1 || g.pbc[k] != 1) cellOk = false;
            g.ncell[k] = std::max(nc, 1);
            cells *= g.ncell[k];
        }
        if (!cellOk || cells > kMaxCells)
            g.ncell[0] = g.ncell[1] = g.ncell[2] = 0;
        g.nimg = (2 * g.pbc[0] + 1) * (2 * g.pbc[1] + 1) * (2 * g.pbc[2] + 1);
        if ((double)n * g.nimg > 2.0e9)
            return fail(err, err_len, N2P2B_ERR_CAPACITY,
                        "n2p2b_neighbor_list_noalloc: too many periodic "
                        "images for this many atoms");
    }
    else
    {
        g.nimg = 1;
    }
    bool const cellPath = g.ncell[0] > 0;
    int const numCells = cellPath ? g.ncell[0] * g.ncell[1] * g.ncell[2] : 0;

    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess)
        return fail(err, err_len, N2P2B_ERR_CUDA,
                    "n2p2b_neighbor_list_noalloc: cannot select the device");
    int* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_address[device])
        {
            void* p = nullptr;
            cudaError_t const e = cudaGetSymbolAddress(&p, g_scratch);
            if (e != cudaSuccess || !p)
            {
                cudaSetDevice(prev);
                return fail(err, err_len, N2P2B_ERR_CUDA,
                            "n2p2b_neighbor_list_noalloc: "
                            "cudaGetSymbolAddress of the scratch failed");
            }
            g_address[device] = static_cast<int*>(p);
        }
        scratch = g_address[device];
    }
    Scratch s;
    s.cellOf = scratch;
    s.cellAtoms = s.cellOf + kMaxAtoms;
    s.cellCount = s.cellAtoms + kMaxAtoms;
    s.cellFill = s.cellCount + (kMaxCells + 1);
    s.cellStart = s.cellFill + (kMaxCells + 1);
    s.status = s.cellStart + (kMaxCells + 1);

    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    int const tb = 256;
    int const gA = (n + tb - 1) / tb;
    int const gW = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
    // Clear what must start at zero (the scratch keeps the last call's data).
    cudaMemsetAsync(s.status, 0, sizeof(int) * kStatusInts, st);
    if (cellPath)
    {
        cudaMemsetAsync(s.cellCount, 0, sizeof(int) * (numCells + 1), st);
        cudaMemsetAsync(s.cellFill, 0, sizeof(int) * (numCells + 1), st);
        naPrepare<<<gA, tb, 0, st>>>(n, g, positions, s);
        naScan<<<1, 1024, 0, st>>>(numCells, s.cellCount, s.cellStart, 0,
                                   s.status, 0);
        naBin<<<gA, tb, 0, st>>>(n, s);
        naCell<0><<<gW, 32 * kWarpsPerBlock, 0, st>>>(
            n, g, positions, s, counts, offsets, index, dr, d);
    }
    naBrute<0><<<gW, 32 * kWarpsPerBlock, 0, st>>>(
        n, g, cellPath ? 1 : 0, positions, s, counts, offsets, index, dr, d);
    naScan<<<1, 1024, 0, st>>>(n, counts, offsets, (long)capacity, s.status, 1);
    if (cellPath)
        naCell<1><<<gW, 32 * kWarpsPerBlock, 0, st>>>(
            n, g, positions, s, counts, offsets, index, dr, d);
    naBrute<1><<<gW, 32 * kWarpsPerBlock, 0, st>>>(
        n, g, cellPath ? 1 : 0, positions, s, counts, offsets, index, dr, d);
    int stat[kStatusInts] = {};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(stat, s.status, sizeof(stat),
                            cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaSetDevice(prev);
    if (e != cudaSuccess)
        return fail(err, err_len, N2P2B_ERR_CUDA, cudaGetErrorString(e));
    *total = (int64_t)(((unsigned long long)(unsigned)stat[S_TOTAL_HI] << 32)
                       | (unsigned long long)(unsigned)stat[S_TOTAL_LO]);
    if ((stat[S_FLAGS] & F_TOO_MANY_NEIGHBORS) && cellPath
        && !(stat[S_FLAGS] & F_OUTSIDE))
        return fail(err, err_len, N2P2B_ERR_CAPACITY,
                    "n2p2b_neighbor_list_noalloc: an atom has more than "
                    "N2P2B_NOALLOC_MAX_NEIGHBORS (1024) neighbors");
    if ((stat[S_FLAGS] & F_OVERFLOW) && *total > 0x7fffffffLL)
        return fail(err, err_len, N2P2B_ERR_CAPACITY,
                    "n2p2b_neighbor_list_noalloc: more than 2^31 - 1 entries "
                    "(int32 offsets); *total holds the number of entries");
    if (stat[S_FLAGS] & F_OVERFLOW)
        return fail(err, err_len, N2P2B_ERR_CAPACITY,
                    "n2p2b_neighbor_list_noalloc: output capacity too small "
                    "(*total holds the required number of entries)");
    return N2P2B_OK;
}
