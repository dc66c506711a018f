// Neighbor list on the device: Structure::remap + Structure::calculateNeighborList
// (libnnp/Structure.cpp:287-399, 1214-1247) with identical neighbor sets.
//
// Bit-exactness.  The reference tests, for every atom pair (i, j) and image
// shift bc in [-pbc, pbc]^3 (pbc from Structure::calculatePbcCopies),
//     dr = r_i - r_j + bc0 * a + bc1 * b + bc2 * c        (Vec3D ops, ISO C++)
//     dr.norm2() <= rc^2,  norm2 = x*x + y*y + z*z
// All products and sums below use __dmul_rn / __dadd_rn / __dsub_rn in that
// association, so no FMA contraction can change a rounding; sqrt is IEEE.
//
// Order.  Each atom's list is stored sorted by the key
//     ((element(j) * N + j) * nimg + img),
//     img = ((bc0 + p0)(2 p1 + 1) + bc1 + p1)(2 p2 + 1) + bc2 + p2
// i.e. grouped by neighbor element and, inside an element, in the reference's
// own (j ascending; bc0, bc1, bc2 ascending) order.  Element grouping gives the
// symmetry-function kernel contiguous per-element neighbor ranges.
//
// Two enumeration paths produce the same set:
//  * cell path: cells at least rc wide along every box vector, 27-cell stencil
//    with periodic wrap.  Used when every box vector's perpendicular width
//    exceeds rc (then pbc = 1) and every atom lies inside the cell (fractional
//    coordinates in [0, 1], true after remap): all neighbors then have
//    |bc| <= 1 and sit in adjacent cells.  Hits are ranked by key per atom.
//  * brute path: all (j, bc) candidates in key order, the reference's own
//    enumeration; used for small or skewed cells, atoms outside the cell and
//    non-periodic structures.
#include "device_common.cuh"
#include "kernels.h"

namespace n2p2b
{

// Structure::remap (libnnp/Structure.cpp:1223-1247) for one atom.
__device__ __forceinline__ void remapAtom(double r[3], double const box[3][3],
                                          double const inv[3][3])
{
    double f[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        f[k] = __dadd_rn(__dadd_rn(__dmul_rn(r[0], inv[0][k]),
                                   __dmul_rn(r[1], inv[1][k])),
                         __dmul_rn(r[2], inv[2][k]));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        if (f[k] > 1.0) f[k] = __dsub_rn(f[k], (double)(int)f[k]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        if (f[k] < 0.0)
            f[k] = __dadd_rn(f[k], __dsub_rn(1.0, (double)(int)f[k]));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        if (f[k] == 1.0) f[k] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        r[k] = __dadd_rn(__dadd_rn(__dmul_rn(f[0], box[0][k]),
                                   __dmul_rn(f[1], box[1][k])),
                         __dmul_rn(f[2], box[2][k]));
    }
}

// Input positions (physical units) -> positions in computing units
// (remap, then Atom::toNormalizedUnits: r *= convLength), plus cell binning.
__global__ void nlPrepareKernel(int n, double const* __restrict__ posIn,
                                int doRemap, int normalize, double convLength,
                                PhysBox pb, NLParams p,
                                double* __restrict__ pos,
                                int* __restrict__ cellOf,
                                int* __restrict__ cellCount,
                                int* __restrict__ status)
{
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double r[3] = {posIn[3 * i + 0], posIn[3 * i + 1], posIn[3 * i + 2]};
    if (doRemap) remapAtom(r, pb.box, pb.invbox);
    if (normalize)
    {
        r[0] = __dmul_rn(r[0], convLength);
        r[1] = __dmul_rn(r[1], convLength);
        r[2] = __dmul_rn(r[2], convLength);
    }
    pos[3 * i + 0] = r[0];
    pos[3 * i + 1] = r[1];
    pos[3 * i + 2] = r[2];
    if (p.ncell[0] > 0)
    {
        int c[3];
        bool inside = true;
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            double const f = r[0] * p.invbox[0][k] + r[1] * p.invbox[1][k]
                           + r[2] * p.invbox[2][k];
            if (!(f >= -1e-12 && f <= 1.0 + 1e-12)) inside = false;
            int ck = (int)floor(f * p.ncell[k]);
            c[k] = min(max(ck, 0), p.ncell[k] - 1);
        }
        if (!inside) atomicOr(&status[ST_FLAGS], FLAG_OUTSIDE_CELL);
        int const cell = (c[0] * p.ncell[1] + c[1]) * p.ncell[2] + c[2];
        cellOf[i] = cell;
        atomicAdd(&cellCount[cell], 1);
    }
}

__global__ void nlBinKernel(int n, int const* __restrict__ cellOf,
                            int const* __restrict__ cellStart,
                            int* __restrict__ cellFill,
                            int* __restrict__ cellAtoms)
{
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int const c = cellOf[i];
    int const slot = atomicAdd(&cellFill[c], 1);
    cellAtoms[cellStart[c] + slot] = i;
}

// Exact reference displacement and cutoff test for candidate (j, bc).
__device__ __forceinline__ bool nlTest(NLParams const& p, double const ri[3],
                                       double const* __restrict__ pos, int j,
                                       int b0, int b1, int b2, double dr[3])
{
    double const db0 = (double)b0, db1 = (double)b1, db2 = (double)b2;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        double v = __dsub_rn(ri[k], pos[3 * j + k]);
        if (p.periodic)
        {
            v = __dadd_rn(v, __dmul_rn(db0, p.box[0][k]));
            v = __dadd_rn(v, __dmul_rn(db1, p.box[1][k]));
            v = __dadd_rn(v, __dmul_rn(db2, p.box[2][k]));
        }
        dr[k] = v;
    }
    double const n2 = __dadd_rn(__dadd_rn(__dmul_rn(dr[0], dr[0]),
                                          __dmul_rn(dr[1], dr[1])),
                                __dmul_rn(dr[2], dr[2]));
    return n2 <= p.rc2;
}

__device__ __forceinline__ int imgIndex(NLParams const& p, int b0, int b1,
                                        int b2)
{
    return ((b0 + p.pbc[0]) * (2 * p.pbc[1] + 1) + (b1 + p.pbc[1]))
           * (2 * p.pbc[2] + 1) + (b2 + p.pbc[2]);
}

__device__ __forceinline__ void imgDecode(NLParams const& p, int img, int& b0,
                                          int& b1, int& b2)
{
    int const n2 = 2 * p.pbc[2] + 1;
    int const n1 = 2 * p.pbc[1] + 1;
    b2 = img % n2 - p.pbc[2];
    img /= n2;
    b1 = img % n1 - p.pbc[1];
    b0 = img / n1 - p.pbc[0];
}

__device__ __forceinline__ unsigned long long nlKey(int ej, int j, int img,
                                                    int n, int nimg)
{
    return ((unsigned long long)ej * (unsigned long long)n
            + (unsigned long long)j) * (unsigned long long)nimg
           + (unsigned long long)img;
}

// Stencil cell c + d (d in {-1,0,1}^3 from s in [0,27)) with periodic wrap;
// returns the cell and the image bc of the atoms found there.
__device__ __forceinline__ int stencilCell(NLParams const& p, int const c[3],
                                           int s, int bc[3])
{
    int const d[3] = {s / 9 - 1, (s / 3) % 3 - 1, s % 3 - 1};
    int cc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        int v = c[k] + d[k];
        int w = 0;
        if (v < 0)                 { v += p.ncell[k]; w = -1; }
        else if (v >= p.ncell[k])  { v -= p.ncell[k]; w = 1; }
        cc[k] = v;
        bc[k] = -w;
    }
    return (cc[0] * p.ncell[1] + cc[1]) * p.ncell[2] + cc[2];
}

// ---------------------------------------------------------------------------
// Cell path.  Warp per atom.  MODE 0 counts hits (total and per element);
// MODE 1 writes the hits' keys, unsorted, into keyTmp[nbrOff[i] ...].
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void nlCellKernel(int n, NLParams p, int numElements,
                             double const* __restrict__ pos,
                             int const* __restrict__ elem,
                             int const* __restrict__ cellOf,
                             int const* __restrict__ cellStart,
                             int const* __restrict__ cellCount,
                             int const* __restrict__ cellAtoms,
                             int* __restrict__ nbrCount,
                             int* __restrict__ nbrCountElem,
                             int const* __restrict__ nbrOff,
                             unsigned long long* __restrict__ keyTmp,
                             int const* __restrict__ status)
{
    if (status[ST_FLAGS] & (FLAG_OUTSIDE_CELL | FLAG_ABORT)) return;
    int const lane = threadIdx.x & 31;
    int const i = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    double const ri[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    int const cell = cellOf[i];
    int c[3];
    c[2] = cell % p.ncell[2];
    c[1] = (cell / p.ncell[2]) % p.ncell[1];
    c[0] = cell / (p.ncell[2] * p.ncell[1]);
    int cntElem[kMaxElem];
#pragma unroll
    for (int e = 0; e < kMaxElem; ++e) cntElem[e] = 0;
    int total = 0;
    long const base = (MODE == 1) ? (long)nbrOff[i] : 0;
    // Lane s < 27 holds stencil cell s (first atom, count, image); the
    // candidates of all 27 cells form one list of `nc` entries that the
    // warp walks 32 at a time, so lanes stay busy across cell boundaries.
    int cs = 0, cn = 0, bcw = 0;
    if (lane < 27)
    {
        int bc[3];
        int const cc = stencilCell(p, c, lane, bc);
        cs = cellStart[cc];
        cn = cellCount[cc];
        bcw = (bc[0] + 1) * 9 + (bc[1] + 1) * 3 + (bc[2] + 1);
    }
    int incl = cn;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        int const v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    int const nc = __shfl_sync(0xffffffffu, incl, 31);
    for (int q0 = 0; q0 < nc; q0 += 32)
    {
        int const q = q0 + lane;
        // Cell of candidate q: the number of cells whose inclusive count
        // end is <= q (ends are nondecreasing over lanes).
        int sc = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1)
        {
            int const probe = sc + step - 1;
            int const v = __shfl_sync(0xffffffffu, incl, probe < 27 ? probe
                                                                    : 26);
            if (probe < 27 && v <= q) sc += step;
        }
        int const src = sc < 27 ? sc : 26;
        int const endS = __shfl_sync(0xffffffffu, incl, src);
        int const cnS = __shfl_sync(0xffffffffu, cn, src);
        int const csS = __shfl_sync(0xffffffffu, cs, src);
        int const bcS = __shfl_sync(0xffffffffu, bcw, src);
        bool hit = false;
        int j = 0;
        int bc[3] = {bcS / 9 - 1, (bcS / 3) % 3 - 1, bcS % 3 - 1};
        int const img = imgIndex(p, bc[0], bc[1], bc[2]);
        if (q < nc)
        {
            j = cellAtoms[csS + (q - (endS - cnS))];
            bool const zeroShift = (bc[0] == 0 && bc[1] == 0 && bc[2] == 0);
            if (!(j == i && zeroShift))
            {
                double dr[3];
                hit = nlTest(p, ri, pos, j, bc[0], bc[1], bc[2], dr);
            }
        }
        {
            unsigned const m = __ballot_sync(0xffffffffu, hit);
            if (MODE == 0)
            {
                if (hit)
                {
                    int const ej = elem[j];
#pragma unroll
                    for (int e = 0; e < kMaxElem; ++e) cntElem[e] += (ej == e);
                }
            }
            else if (hit)
            {
                int const off = total + __popc(m & ((1u << lane) - 1u));
                keyTmp[base + off] = nlKey(elem[j], j, img, n, p.nimg);
            }
            total += __popc(m);
        }
    }
    if (MODE == 0)
    {
        for (int e = 0; e < numElements; ++e)
        {
            int v = cntElem[e];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) nbrCountElem[(long)i * numElements + e] = v;
        }
        if (lane == 0) nbrCount[i] = total;
    }
}

// ---------------------------------------------------------------------------
// Brute path.  Warp per atom, candidates enumerated in key order:
// element-major, then j ascending (atomsByElem is sorted per element), then
// image.  MODE 0 counts; MODE 1 writes keys (already sorted) into key[].
// `onlyIfOutside`: the cell path was eligible, so run only if some atom was
// found outside the cell.
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void nlBruteKernel(int n, NLParams p, int numElements,
                              int onlyIfOutside,
                              double const* __restrict__ pos,
                              int const* __restrict__ atomsByElem,
                              ElemStarts es,
                              int* __restrict__ nbrCount,
                              int* __restrict__ nbrCountElem,
                              int const* __restrict__ nbrOff,
                              unsigned long long* __restrict__ key,
                              int const* __restrict__ status)
{
    int const flags = status[ST_FLAGS];
    if (flags & FLAG_ABORT) return;
    if (onlyIfOutside && !(flags & FLAG_OUTSIDE_CELL)) return;
    int const lane = threadIdx.x & 31;
    int const i = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    double const ri[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    int total = 0;
    long const base = (MODE == 1) ? (long)nbrOff[i] : 0;
    int const nimg = p.nimg;
    for (int e = 0; e < numElements; ++e)
    {
        int const eb = es.start[e];
        long const ncand = (long)(es.start[e + 1] - eb) * nimg;
        int cntE = 0;
        for (long c0 = 0; c0 < ncand; c0 += 32)
        {
            long const c = c0 + lane;
            bool hit = false;
            int j = 0, img = 0;
            if (c < ncand)
            {
                j = atomsByElem[eb + (int)(c / nimg)];
                img = (int)(c % nimg);
                int b0, b1, b2;
                imgDecode(p, img, b0, b1, b2);
                if (!(j == i && b0 == 0 && b1 == 0 && b2 == 0))
                {
                    double dr[3];
                    hit = nlTest(p, ri, pos, j, b0, b1, b2, dr);
                }
            }
            unsigned const m = __ballot_sync(0xffffffffu, hit);
            if (MODE == 1 && hit)
            {
                int const off = total + __popc(m & ((1u << lane) - 1u));
                key[base + off] = nlKey(e, j, img, n, nimg);
            }
            total += __popc(m);
            cntE += __popc(m);
        }
        if (MODE == 0 && lane == 0)
            nbrCountElem[(long)i * numElements + e] = cntE;
    }
    if (MODE == 0 && lane == 0) nbrCount[i] = total;
}

// Exclusive scan of per-atom counts into offsets (n + 1 entries), total and
// maximum into the status words; flags overflow against `capacity`.
// Single block; each thread scans a contiguous chunk.
__global__ void nlScanKernel(int n, int const* __restrict__ cnt,
                             int* __restrict__ off, long capacity,
                             int* __restrict__ status)
{
    __shared__ long sPart[1024];
    __shared__ int sMax[1024];
    int const t = threadIdx.x;
    int const T = blockDim.x;
    int const chunk = (n + T - 1) / T;
    int const b = min(n, t * chunk);
    int const e = min(n, b + chunk);
    long s = 0;
    int mx = 0;
    for (int i = b; i < e; ++i)
    {
        s += cnt[i];
        mx = max(mx, cnt[i]);
    }
    sPart[t] = s;
    sMax[t] = mx;
    __syncthreads();
    if (t == 0)
    {
        long run = 0;
        int m = 0;
        for (int k = 0; k < T; ++k)
        {
            long const v = sPart[k];
            sPart[k] = run;
            run += v;
            m = max(m, sMax[k]);
        }
        off[n] = (int)min(run, (long)0x7fffffff);
        status[ST_TOTAL_NBR] = (int)min(run, (long)0x7fffffff);
        status[ST_MAX_NBR] = m;
        if (run > capacity)
        {
            status[ST_FLAGS] |= FLAG_NBR_OVERFLOW | FLAG_ABORT;
        }
    }
    __syncthreads();
    long run = sPart[t];
    for (int i = b; i < e; ++i)
    {
        off[i] = (int)run;
        run += cnt[i];
    }
}

// Warp per atom: (cell path) rank the unsorted keys; then decode every entry
// into the structure-of-arrays neighbor list with the exact displacement.
__global__ void nlFinishKernel(int n, NLParams p, int sortKeys,
                               double const* __restrict__ pos,
                               int const* __restrict__ elem,
                               int const* __restrict__ nbrOff,
                               unsigned long long const* __restrict__ keyTmp,
                               unsigned long long* __restrict__ key,
                               int* __restrict__ nbrIdx,
                               int8_t* __restrict__ nbrEl,
                               double* __restrict__ dx,
                               double* __restrict__ dy,
                               double* __restrict__ dz,
                               double* __restrict__ dd,
                               int const* __restrict__ status)
{
    int const flags = status[ST_FLAGS];
    if (flags & FLAG_ABORT) return;
    // The cell path's keys are only valid if it ran.
    if (sortKeys && (flags & FLAG_OUTSIDE_CELL)) sortKeys = 0;
    int const lane = threadIdx.x & 31;
    int const i = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    long const b = nbrOff[i];
    int const cnt = nbrOff[i + 1] - nbrOff[i];
    if (sortKeys)
    {
        for (int t = lane; t < cnt; t += 32)
        {
            unsigned long long const k = keyTmp[b + t];
            int r = 0;
            for (int u = 0; u < cnt; ++u) r += (keyTmp[b + u] < k);
            key[b + r] = k;
        }
        __syncwarp();
    }
    double const ri[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    unsigned long long const nimg = (unsigned long long)p.nimg;
    for (int t = lane; t < cnt; t += 32)
    {
        unsigned long long const k = key[b + t];
        int const img = (int)(k % nimg);
        unsigned long long const q = k / nimg;
        int const j = (int)(q % (unsigned long long)n);
        int b0, b1, b2;
        imgDecode(p, img, b0, b1, b2);
        double dr[3];
        nlTest(p, ri, pos, j, b0, b1, b2, dr);
        double const n2 = __dadd_rn(__dadd_rn(__dmul_rn(dr[0], dr[0]),
                                              __dmul_rn(dr[1], dr[1])),
                                    __dmul_rn(dr[2], dr[2]));
        nbrIdx[b + t] = j;
        nbrEl[b + t] = (int8_t)elem[j];
        dx[b + t] = dr[0];
        dy[b + t] = dr[1];
        dz[b + t] = dr[2];
        dd[b + t] = __dsqrt_rn(n2);
    }
}

// Thread per entry: position of the mirror entry (j -> i, -bc) in j's list,
// found by binary search over j's sorted keys.  Exists by symmetry: IEEE
// rounding is sign-symmetric, so the mirror displacement is exactly -dr.
__global__ void nlMirrorKernel(int n, int nimg,
                               int const* __restrict__ elem,
                               int const* __restrict__ nbrOff,
                               unsigned long long const* __restrict__ key,
                               int const* __restrict__ nbrIdx,
                               int const* __restrict__ entryAtom,
                               int* __restrict__ mirror,
                               int* __restrict__ status)
{
    if (status[ST_FLAGS] & FLAG_ABORT) return;
    long const e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)nbrOff[n]) return;
    int const i = entryAtom[e];
    int const j = nbrIdx[e];
    unsigned long long const nimgU = (unsigned long long)nimg;
    int const img = (int)(key[e] % nimgU);
    unsigned long long const want = nlKey(elem[i], i, nimg - 1 - img, n, nimg);
    long lo = nbrOff[j], hi = nbrOff[j + 1];
    while (lo < hi)
    {
        long const mid = (lo + hi) >> 1;
        if (key[mid] < want) lo = mid + 1;
        else hi = mid;
    }
    if (lo < nbrOff[j + 1] && key[lo] == want)
    {
        mirror[e] = (int)lo;
    }
    else
    {
        mirror[e] = -1;
        atomicOr(&status[ST_FLAGS], FLAG_MIRROR_MISSING);
    }
}

// Thread per atom: owner atom of every entry (for entry-parallel kernels).
__global__ void nlEntryAtomKernel(int n, int const* __restrict__ nbrOff,
                                  int* __restrict__ entryAtom,
                                  int const* __restrict__ status)
{
    if (status[ST_FLAGS] & FLAG_ABORT) return;
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int e = nbrOff[i]; e < nbrOff[i + 1]; ++e) entryAtom[e] = i;
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------

void launchNeighborList(NLLaunch const& L, cudaStream_t s)
{
    int const n = L.n;
    int const tb = 256;
    int const gAtoms = (n + tb - 1) / tb;
    int const warpsPerBlock = 4;
    int const gWarp = (n + warpsPerBlock - 1) / warpsPerBlock;
    bool const cellEligible = L.p.ncell[0] > 0;
    if (cellEligible)
    {
        cudaMemsetAsync(L.cellCount, 0, sizeof(int) * (size_t)L.numCells, s);
        cudaMemsetAsync(L.cellFill, 0, sizeof(int) * (size_t)L.numCells, s);
    }
    nlPrepareKernel<<<gAtoms, tb, 0, s>>>(n, L.posIn, L.doRemap, L.normalize,
                                          L.convLength, L.pb, L.p, L.pos,
                                          L.cellOf, L.cellCount, L.status);
    if (cellEligible)
    {
        nlScanKernel<<<1, 1024, 0, s>>>(L.numCells, L.cellCount, L.cellStart,
                                        0x7fffffffL, L.cellScanStatus);
        nlBinKernel<<<gAtoms, tb, 0, s>>>(n, L.cellOf, L.cellStart,
                                          L.cellFill, L.cellAtoms);
        nlCellKernel<0><<<gWarp, 32 * warpsPerBlock, 0, s>>>(
            n, L.p, L.numElements, L.pos, L.elem, L.cellOf, L.cellStart,
            L.cellCount, L.cellAtoms, L.nbrCount, L.nbrCountElem, L.nbrOff,
            L.keyTmp, L.status);
    }
    nlBruteKernel<0><<<gWarp, 32 * warpsPerBlock, 0, s>>>(
        n, L.p, L.numElements, cellEligible ? 1 : 0, L.pos, L.atomsByElem,
        L.es, L.nbrCount, L.nbrCountElem, L.nbrOff, L.key, L.status);
    nlScanKernel<<<1, 1024, 0, s>>>(n, L.nbrCount, L.nbrOff, L.capacity,
                                    L.status);
    if (cellEligible)
    {
        nlCellKernel<1><<<gWarp, 32 * warpsPerBlock, 0, s>>>(
            n, L.p, L.numElements, L.pos, L.elem, L.cellOf, L.cellStart,
            L.cellCount, L.cellAtoms, L.nbrCount, L.nbrCountElem, L.nbrOff,
            L.keyTmp, L.status);
    }
    nlBruteKernel<1><<<gWarp, 32 * warpsPerBlock, 0, s>>>(
        n, L.p, L.numElements, cellEligible ? 1 : 0, L.pos, L.atomsByElem,
        L.es, L.nbrCount, L.nbrCountElem, L.nbrOff, L.key, L.status);
    nlFinishKernel<<<gWarp, 32 * warpsPerBlock, 0, s>>>(
        n, L.p, cellEligible ? 1 : 0, L.pos, L.elem, L.nbrOff, L.keyTmp,
        L.key, L.nbrIdx, L.nbrEl, L.dx, L.dy, L.dz, L.dd, L.status);
    nlEntryAtomKernel<<<gAtoms, tb, 0, s>>>(n, L.nbrOff, L.entryAtom,
                                            L.status);
    long const cap = L.capacity;
    int const gE = (int)((cap + tb - 1) / tb);
    noteLaunches(cellEligible ? 11 : 7);
    nlMirrorKernel<<<gE > 0 ? gE : 1, tb, 0, s>>>(
        n, L.p.nimg, L.elem, L.nbrOff, L.key, L.nbrIdx,
        L.entryAtom, L.mirror, L.status);
}

// ===========================================================================
// Batches of independent structures (one neighbor list per structure, all
// structures' atoms concatenated).  Every structure keeps its own box and
// image range; candidates are the atoms of the same structure only, in the
// brute path's key order, so each structure's list is exactly the one
// Structure::calculateNeighborList builds for it alone.  Keys use the
// batch-wide image stride NIMG (the largest structure's image count) so
// that they stay unique and sorted.
// ===========================================================================

__global__ void nlbPrepareKernel(int n, double const* __restrict__ posIn,
                                 int const* __restrict__ structOf,
                                 BatchStruct const* __restrict__ bs,
                                 int normalize, double convLength,
                                 double* __restrict__ pos)
{
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    BatchStruct const& S = bs[structOf[i]];
    double r[3] = {posIn[3 * i + 0], posIn[3 * i + 1], posIn[3 * i + 2]};
    if (S.doRemap) remapAtom(r, S.pb.box, S.pb.invbox);
    if (normalize)
    {
        r[0] = __dmul_rn(r[0], convLength);
        r[1] = __dmul_rn(r[1], convLength);
        r[2] = __dmul_rn(r[2], convLength);
    }
    pos[3 * i + 0] = r[0];
    pos[3 * i + 1] = r[1];
    pos[3 * i + 2] = r[2];
}

// Warp per atom; MODE 0 counts, MODE 1 writes the (sorted) keys.
template <int MODE>
__global__ void nlbBruteKernel(int n, int numElements, int NIMG,
                               double const* __restrict__ pos,
                               int const* __restrict__ structOf,
                               BatchStruct const* __restrict__ bs,
                               int const* __restrict__ structAtoms,
                               int* __restrict__ nbrCount,
                               int* __restrict__ nbrCountElem,
                               int const* __restrict__ nbrOff,
                               unsigned long long* __restrict__ key,
                               int const* __restrict__ status)
{
    if (status[ST_FLAGS] & FLAG_ABORT) return;
    int const lane = threadIdx.x & 31;
    int const i = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    BatchStruct const& S = bs[structOf[i]];
    NLParams const& p = S.p;
    double const ri[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    int total = 0;
    long const base = (MODE == 1) ? (long)nbrOff[i] : 0;
    int const nimg = p.nimg;
    for (int e = 0; e < numElements; ++e)
    {
        int const eb = S.es[e];
        long const ncand = (long)(S.es[e + 1] - eb) * nimg;
        int cntE = 0;
        for (long c0 = 0; c0 < ncand; c0 += 32)
        {
            long const c = c0 + lane;
            bool hit = false;
            int j = 0, img = 0;
            if (c < ncand)
            {
                j = structAtoms[eb + (int)(c / nimg)];
                img = (int)(c % nimg);
                int b0, b1, b2;
                imgDecode(p, img, b0, b1, b2);
                if (!(j == i && b0 == 0 && b1 == 0 && b2 == 0))
                {
                    double dr[3];
                    hit = nlTest(p, ri, pos, j, b0, b1, b2, dr);
                }
            }
            unsigned const m = __ballot_sync(0xffffffffu, hit);
            if (MODE == 1 && hit)
            {
                int const off = total + __popc(m & ((1u << lane) - 1u));
                key[base + off] = nlKey(e, j, img, n, NIMG);
            }
            total += __popc(m);
            cntE += __popc(m);
        }
        if (MODE == 0 && lane == 0)
            nbrCountElem[(long)i * numElements + e] = cntE;
    }
    if (MODE == 0 && lane == 0) nbrCount[i] = total;
}

__global__ void nlbFinishKernel(int n, int NIMG,
                                double const* __restrict__ pos,
                                int const* __restrict__ elem,
                                int const* __restrict__ structOf,
                                BatchStruct const* __restrict__ bs,
                                int const* __restrict__ nbrOff,
                                unsigned long long const* __restrict__ key,
                                int* __restrict__ nbrIdx,
                                int8_t* __restrict__ nbrEl,
                                double* __restrict__ dx,
                                double* __restrict__ dy,
                                double* __restrict__ dz,
                                double* __restrict__ dd,
                                int const* __restrict__ status)
{
    if (status[ST_FLAGS] & FLAG_ABORT) return;
    int const lane = threadIdx.x & 31;
    int const i = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    NLParams const& p = bs[structOf[i]].p;
    long const b = nbrOff[i];
    int const cnt = nbrOff[i + 1] - nbrOff[i];
    double const ri[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    unsigned long long const nimg = (unsigned long long)NIMG;
    for (int t = lane; t < cnt; t += 32)
    {
        unsigned long long const k = key[b + t];
        int const img = (int)(k % nimg);
        int const j = (int)((k / nimg) % (unsigned long long)n);
        int b0, b1, b2;
        imgDecode(p, img, b0, b1, b2);
        double dr[3];
        nlTest(p, ri, pos, j, b0, b1, b2, dr);
        double const n2 = __dadd_rn(__dadd_rn(__dmul_rn(dr[0], dr[0]),
                                              __dmul_rn(dr[1], dr[1])),
                                    __dmul_rn(dr[2], dr[2]));
        nbrIdx[b + t] = j;
        nbrEl[b + t] = (int8_t)elem[j];
        dx[b + t] = dr[0];
        dy[b + t] = dr[1];
        dz[b + t] = dr[2];
        dd[b + t] = __dsqrt_rn(n2);
    }
}

__global__ void nlbMirrorKernel(int n, int NIMG,
                                int const* __restrict__ elem,
                                int const* __restrict__ structOf,
                                BatchStruct const* __restrict__ bs,
                                int const* __restrict__ nbrOff,
                                unsigned long long const* __restrict__ key,
                                int const* __restrict__ nbrIdx,
                                int const* __restrict__ entryAtom,
                                int* __restrict__ mirror,
                                int* __restrict__ status)
{
    if (status[ST_FLAGS] & FLAG_ABORT) return;
    long const e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)nbrOff[n]) return;
    int const i = entryAtom[e];
    int const j = nbrIdx[e];
    int const nimg = bs[structOf[i]].p.nimg;
    int const img = (int)(key[e] % (unsigned long long)NIMG);
    unsigned long long const want = nlKey(elem[i], i, nimg - 1 - img, n, NIMG);
    long lo = nbrOff[j], hi = nbrOff[j + 1];
    while (lo < hi)
    {
        long const mid = (lo + hi) >> 1;
        if (key[mid] < want) lo = mid + 1;
        else hi = mid;
    }
    if (lo < nbrOff[j + 1] && key[lo] == want)
    {
        mirror[e] = (int)lo;
    }
    else
    {
        mirror[e] = -1;
        atomicOr(&status[ST_FLAGS], FLAG_MIRROR_MISSING);
    }
}

// Batch neighbor list, faster form of nlbBruteKernel for structures with at
// most 128 images (|bc| <= 2 per box vector): warp per atom i, lanes over
// the candidates j of one element (positions loaded once), each lane walks
// the structure's images in key order with an incremental (b0, b1, b2)
// counter.  An FP32 distance test only filters: its threshold rc^2 + m
// covers the FP32 rounding of the displacement and image-shift sums (m from
// a bound on their magnitudes, at least 1e-4 rc^2), and every candidate it
// keeps gets the exact FP64 test of nlTest, so the neighbor sets are those
// of the brute path.  Hits are kept
// as per-lane image bit masks and written in key order (lane = j
// ascending, bits = image ascending) through a warp prefix sum.
template <int MODE>
__global__ void nlbLaneKernel(int n, int numElements, int NIMG,
                              double const* __restrict__ pos,
                              int const* __restrict__ structOf,
                              BatchStruct const* __restrict__ bs,
                              int const* __restrict__ structAtoms,
                              int* __restrict__ nbrCount,
                              int* __restrict__ nbrCountElem,
                              int const* __restrict__ nbrOff,
                              unsigned long long* __restrict__ key,
                              int const* __restrict__ status)
{
    if (status[ST_FLAGS] & FLAG_ABORT) return;
    int const lane = threadIdx.x & 31;
    int const i = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    BatchStruct const& S = bs[structOf[i]];
    NLParams const& p = S.p;
    int const nimg = p.nimg;
    int const q0 = p.periodic ? p.pbc[0] : 0;
    int const q1 = p.periodic ? p.pbc[1] : 0;
    int const q2 = p.periodic ? p.pbc[2] : 0;
    float a[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) a[r][c] = (float)p.box[r][c];
    double const ri[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    // Largest image shift per component: sum_r |pbc_r a_r|.
    float shiftMax = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        shiftMax = fmaxf(shiftMax, fabsf(a[0][c]) * q0 + fabsf(a[1][c]) * q1
                                   + fabsf(a[2][c]) * q2);
    float const rcf = sqrtf((float)p.rc2);
    int total = 0;
    long const base = (MODE == 1) ? (long)nbrOff[i] : 0;
    for (int e = 0; e < numElements; ++e)
    {
        int const eb = S.es[e];
        int const ne = S.es[e + 1] - eb;
        int cntE = 0;
        for (int j0 = 0; j0 < ne; j0 += 32)
        {
            int const jj = j0 + lane;
            unsigned mask[4] = {0u, 0u, 0u, 0u};
            int j = 0;
            if (jj < ne)
            {
                j = structAtoms[eb + jj];
                float const d0 = (float)(ri[0] - pos[3 * j + 0]);
                float const d1 = (float)(ri[1] - pos[3 * j + 1]);
                float const d2 = (float)(ri[2] - pos[3 * j + 2]);
                // Per component the FP32 sum of up to four terms of size
                // <= M errs by < 8 M 2^-24 (rounded box included); r^2
                // near the cutoff then errs by < 2 rc 3 e + 3 e^2.
                float const M = fmaxf(fmaxf(fabsf(d0), fabsf(d1)), fabsf(d2))
                              + shiftMax;
                float const err = 8.0f * M * 5.9604645e-8f;
                float const rc2f = (float)p.rc2
                                 + fmaxf(1e-4f * (float)p.rc2,
                                         4.0f * (6.0f * rcf * err
                                                 + 3.0f * err * err));
                int b0 = -q0, b1 = -q1, b2 = -q2;
                for (int img = 0; img < nimg; ++img)
                {
                    float const x = d0 + b0 * a[0][0] + b1 * a[1][0]
                                  + b2 * a[2][0];
                    float const y = d1 + b0 * a[0][1] + b1 * a[1][1]
                                  + b2 * a[2][1];
                    float const z = d2 + b0 * a[0][2] + b1 * a[1][2]
                                  + b2 * a[2][2];
                    if (x * x + y * y + z * z <= rc2f
                        && !(j == i && b0 == 0 && b1 == 0 && b2 == 0))
                    {
                        double dr[3];
                        if (nlTest(p, ri, pos, j, b0, b1, b2, dr))
                            mask[img >> 5] |= 1u << (img & 31);
                    }
                    if (++b2 > q2)
                    {
                        b2 = -q2;
                        if (++b1 > q1)
                        {
                            b1 = -q1;
                            ++b0;
                        }
                    }
                }
            }
            int const c = __popc(mask[0]) + __popc(mask[1]) + __popc(mask[2])
                        + __popc(mask[3]);
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                int const v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            int const sum = __shfl_sync(0xffffffffu, incl, 31);
            if (MODE == 1 && c > 0)
            {
                int off = total + incl - c;
                for (int w = 0; w < 4; ++w)
                {
                    unsigned m = mask[w];
                    while (m)
                    {
                        int const img = (w << 5) + __ffs(m) - 1;
                        m &= m - 1;
                        key[base + off++] = nlKey(e, j, img, n, NIMG);
                    }
                }
            }
            total += sum;
            cntE += sum;
        }
        if (MODE == 0 && lane == 0)
            nbrCountElem[(long)i * numElements + e] = cntE;
    }
    if (MODE == 0 && lane == 0) nbrCount[i] = total;
}

void launchNeighborListBatch(NLBatchLaunch const& L, cudaStream_t s)
{
    int const n = L.n;
    int const tb = 256;
    int const gAtoms = (n + tb - 1) / tb;
    int const wpb = L.warpsPerBlock > 0 ? L.warpsPerBlock : 4;
    int const gWarp = (n + wpb - 1) / wpb;
    nlbPrepareKernel<<<gAtoms, tb, 0, s>>>(n, L.posIn, L.structOf, L.bs,
                                           L.normalize, L.convLength, L.pos);
    // Structures with more than 128 images (boxes below rc / 2) take the
    // plain brute path.
    if (L.NIMG <= 128)
    {
        nlbLaneKernel<0><<<gWarp, 32 * wpb, 0, s>>>(
            n, L.numElements, L.NIMG, L.pos, L.structOf, L.bs,
            L.structAtoms, L.nbrCount, L.nbrCountElem, L.nbrOff, L.key,
            L.status);
        nlScanKernel<<<1, 1024, 0, s>>>(n, L.nbrCount, L.nbrOff, L.capacity,
                                        L.status);
        nlbLaneKernel<1><<<gWarp, 32 * wpb, 0, s>>>(
            n, L.numElements, L.NIMG, L.pos, L.structOf, L.bs,
            L.structAtoms, L.nbrCount, L.nbrCountElem, L.nbrOff, L.key,
            L.status);
    }
    else
    {
        nlbBruteKernel<0><<<gWarp, 32 * wpb, 0, s>>>(
            n, L.numElements, L.NIMG, L.pos, L.structOf, L.bs,
            L.structAtoms, L.nbrCount, L.nbrCountElem, L.nbrOff, L.key,
            L.status);
        nlScanKernel<<<1, 1024, 0, s>>>(n, L.nbrCount, L.nbrOff, L.capacity,
                                        L.status);
        nlbBruteKernel<1><<<gWarp, 32 * wpb, 0, s>>>(
            n, L.numElements, L.NIMG, L.pos, L.structOf, L.bs,
            L.structAtoms, L.nbrCount, L.nbrCountElem, L.nbrOff, L.key,
            L.status);
    }
    nlbFinishKernel<<<gWarp, 32 * wpb, 0, s>>>(
        n, L.NIMG, L.pos, L.elem, L.structOf, L.bs, L.nbrOff, L.key,
        L.nbrIdx, L.nbrEl, L.dx, L.dy, L.dz, L.dd, L.status);
    nlEntryAtomKernel<<<gAtoms, tb, 0, s>>>(n, L.nbrOff, L.entryAtom,
                                            L.status);
    long const cap = L.capacity;
    int const gE = (int)((cap + tb - 1) / tb);
    noteLaunches(7);
    nlbMirrorKernel<<<gE > 0 ? gE : 1, tb, 0, s>>>(
        n, L.NIMG, L.elem, L.structOf, L.bs, L.nbrOff, L.key, L.nbrIdx,
        L.entryAtom, L.mirror, L.status);
}

} // namespace n2p2b
