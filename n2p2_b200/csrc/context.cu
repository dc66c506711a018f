// Context: owns the potential, the device tables and the device buffers of
// one structure, and runs the prediction pipeline behind the C-ABI
// (include/n2p2_b200.h).  Host-side geometry (inverse box, periodic image
// counts) is computed with the reference's own expressions; this file is
// compiled with -ffp-contract=off for its host code so those roundings match.
#include "n2p2_b200.h"

#include "kernels.h"
#include "potential.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <map>
#include <vector>

using namespace n2p2b;

namespace
{

struct CudaError : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

struct CapacityError : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

struct StateError : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

struct ExtrapolationError : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, char const* what)
{
    if (e != cudaSuccess)
    {
        throw CudaError(std::string("CUDA error in ") + what + ": "
                        + cudaGetErrorString(e));
    }
}

// Grow-only device allocation.
struct DevBuf
{
    void*       p = nullptr;
    std::size_t bytes = 0;
    void ensure(std::size_t b)
    {
        if (b <= bytes && p != nullptr) return;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        std::size_t const want = std::max<std::size_t>(b, 256);
        ck(cudaMalloc(&p, want), "cudaMalloc");
        bytes = want;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// --- reference geometry (libnnp/Vec3D.h, Structure.cpp) --------------------

struct V3
{
    double r[3];
};

V3 cross(V3 const& a, V3 const& b)
{
    V3 w;
    w.r[0] = a.r[1] * b.r[2] - a.r[2] * b.r[1];
    w.r[1] = a.r[2] * b.r[0] - a.r[0] * b.r[2];
    w.r[2] = a.r[0] * b.r[1] - a.r[1] * b.r[0];
    return w;
}

V3 normalized(V3 v)
{
    double const n = std::sqrt(v.r[0] * v.r[0] + v.r[1] * v.r[1]
                               + v.r[2] * v.r[2]);
    v.r[0] /= n;
    v.r[1] /= n;
    v.r[2] /= n;
    return v;
}

double dot(V3 const& a, V3 const& b)
{
    return a.r[0] * b.r[0] + a.r[1] * b.r[1] + a.r[2] * b.r[2];
}

// Structure::calculateInverseBox (libnnp/Structure.cpp:519-546).
void inverseBox(double const box[3][3], double inv[3][3])
{
    double invdet = box[0][0] * box[1][1] * box[2][2]
                  + box[1][0] * box[2][1] * box[0][2]
                  + box[2][0] * box[0][1] * box[1][2]
                  - box[2][0] * box[1][1] * box[0][2]
                  - box[0][0] * box[2][1] * box[1][2]
                  - box[1][0] * box[0][1] * box[2][2];
    invdet = 1.0 / invdet;
    inv[0][0] = box[1][1] * box[2][2] - box[2][1] * box[1][2];
    inv[0][1] = box[2][1] * box[0][2] - box[0][1] * box[2][2];
    inv[0][2] = box[0][1] * box[1][2] - box[1][1] * box[0][2];
    inv[1][0] = box[2][0] * box[1][2] - box[1][0] * box[2][2];
    inv[1][1] = box[0][0] * box[2][2] - box[2][0] * box[0][2];
    inv[1][2] = box[1][0] * box[0][2] - box[0][0] * box[1][2];
    inv[2][0] = box[1][0] * box[2][1] - box[2][0] * box[1][1];
    inv[2][1] = box[2][0] * box[0][1] - box[0][0] * box[2][1];
    inv[2][2] = box[0][0] * box[1][1] - box[1][0] * box[0][1];
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c) inv[k][c] *= invdet;
}

// Structure::calculatePbcCopies (libnnp/Structure.cpp:486-517); also returns
// the perpendicular widths used for the cell grid.
void pbcCopies(double const box[3][3], double rc, int pbc[3], double proj[3])
{
    V3 a{{box[0][0], box[0][1], box[0][2]}};
    V3 b{{box[1][0], box[1][1], box[1][2]}};
    V3 c{{box[2][0], box[2][1], box[2][2]}};
    V3 const axb = normalized(cross(a, b));
    V3 const axc = normalized(cross(a, c));
    V3 const bxc = normalized(cross(b, c));
    proj[0] = std::fabs(dot(a, bxc));
    proj[1] = std::fabs(dot(b, axc));
    proj[2] = std::fabs(dot(c, axb));
    for (int k = 0; k < 3; ++k)
    {
        pbc[k] = 0;
        while (pbc[k] * proj[k] <= rc) pbc[k]++;
    }
}

__global__ void statusResetKernel(int* status)
{
    if (threadIdx.x < ST_NUM) status[threadIdx.x] = 0;
    if (threadIdx.x == ST_BAD_ATOM) status[threadIdx.x] = -1;
}

std::atomic<unsigned long long> g_launches{0};

// Stage boundaries of one profiled pipeline run: events before NL and after
// NL, SF, NN, energy and forces (stages not run record nothing).
struct StageEvents
{
    cudaEvent_t ev[6];
    bool        used[6];
};

} // namespace

namespace n2p2b
{
void noteLaunches(int k) { g_launches += (unsigned long long)k; }
} // namespace n2p2b

struct n2p2b_context
{
    int          device = 0;
    cudaStream_t stream = nullptr;
    bool         ownStream = false;
    std::string  error;

    // Potential and its device tables.
    Potential    pot;
    bool         generic = false;
    bool         scaled = false;
    bool         weighted = false;
    bool         tablesReady = false;
    SFParams     sfp{};
    std::vector<DevGroup>  tabGroups;    // SF tables (sfp points here)
    std::vector<DevMember> tabMembers;
    DevBuf       tabGroupsDev, tabMembersDev;
    NNParams     nnp{};
    int          maxSF = 0;
    int          maxSlots = 0;
    DevBuf       sfScale, nnW, slotSF;
    // Mixed forms (FP32 symmetry functions, BF16 tensor-core NNs); index 0
    // = PREC_BF16 (hi/lo operands in the forward sweep and for dE/dG, single
    // BF16 deltas with hi/lo weights in the other backward GEMMs: 2 MMAs per
    // K-step there), 1 = PREC_MIXED (hi/lo operands everywhere: 3 MMAs).
    int          precision = PREC_FP64;
    TcNNParams   tcp[2] = {};
    bool         tcOk[2] = {false, false};
    std::string  tcWhy[2];
    DevBuf       tcW[2], tcF[2];
    int          tcGrid[2] = {0, 0};
    // Extrapolation warnings (Mode::setupSymmetryFunctionStatistics).
    bool         ewCheck = false, ewWrite = false, ewStop = false;
    long         ewTotal = 0;
    bool         haveEW = false;
    std::vector<Range> ewRangeHost;
    std::vector<SFScale> sfScaleHost;
    DevBuf       ewRange, ewPerAtom;

    // Externally supplied neighbor list (n2p2b_set_neighbor_list).
    bool         externalNL = false;
    long         numTargets = 0;
    DevBuf       revOff, revEntry, Ftarget;

    // Batch of independent structures (numStructs > 0).
    long         numStructs = 0;
    int          batchNIMG = 1;
    std::vector<BatchStruct> bsHost;
    std::vector<int64_t> structCounts;
    DevBuf       structOf, structAtoms, bsDev, structEnergy;
    int          nlWarpsPerBlock = 4;

    // CUDA graph of one whole evaluation (n2p2b_capture_graph).
    bool            graphValid = false;
    bool            graphForces = true;
    cudaGraphExec_t graphExec = nullptr;

    // Distilled student network (FP32, same symmetry functions).
    struct Student
    {
        bool               loaded = false;
        Potential          pot;
        NNParams           nnp{};
        std::vector<float> blob;
        int                mode = 0;         // 0 off, 1 gated, 2 student only
        bool               trainable = false;
        std::string        whyNot;
        std::vector<Range> range;            // training range (unscaled)
        bool               haveRange = false;
        long               step = 0;         // Adam steps taken
        int                maxH = 0, maxNin = 0, maxParams = 0;
        DevBuf             w, m, v, grad, gpart, rE, rF, u, loss, dRange,
                           list, listCount, lrScale;
    } stu;

    // Structure.
    long         n = 0;
    bool         periodic = false;
    bool         remap = false;
    double       boxPhys[3][3] = {};
    std::vector<int32_t> elemHost;
    NLParams     nlp{};
    PhysBox      pb{};
    ElemStarts   es{};
    int          numCells = 0;
    DevBuf       posIn, pos, elem, atomsByElem;
    DevBuf       cellOf, cellCount, cellFill, cellStart, cellAtoms, cellStatus;
    DevBuf       nbrCount, nbrCountElem, nbrOff;
    long         capacity = 0;
    DevBuf       keyTmp, key, nbrIdx, nbrEl, dx, dy, dz, dd, entryAtom, mirror;
    DevBuf       pairF, dGdr;
    DevBuf       G, dEdG, dGdrSelf, Ei, selfF, F, energyOut, status;
    int*         statusHost = nullptr;
    double*      energyHost = nullptr;
    int          sfCap = 0;      // 0 = size from the next neighbor list
    int          lastMaxNbr = 0; // largest neighbor count of the last list
    int          sfGrid = 0;
    int          sfGridCap = 0;
    int          sfVariant = -1;  // chosen from the potential's groups
    int          sfSortCats = 0;
    int          smCount = 0;

    // Pipeline state (what the last calls computed).
    bool haveNL = false, haveSF = false, haveSFDeriv = false, haveNN = false;
    bool haveNNDeriv = false, haveE = false, haveF = false;

    // Per-stage device timing (n2p2b_set_profiling).
    bool                     profiling = false;
    std::vector<StageEvents> pendingEvents;
    std::vector<StageEvents> freeEvents;
    double                   stageMs[5] = {0, 0, 0, 0, 0};
    long                     stageRuns = 0;
    StageEvents*             cur = nullptr;

    void mark(int k)
    {
        if (!cur) return;
        ck(cudaEventRecord(cur->ev[k], stream), "cudaEventRecord");
        cur->used[k] = true;
    }

    void beginProfile()
    {
        if (!profiling) return;
        StageEvents se;
        if (!freeEvents.empty())
        {
            se = freeEvents.back();
            freeEvents.pop_back();
        }
        else
        {
            for (auto& e : se.ev) ck(cudaEventCreate(&e), "cudaEventCreate");
        }
        for (auto& u : se.used) u = false;
        pendingEvents.push_back(se);
        cur = &pendingEvents.back();
        mark(0);
    }

    void endProfile() { cur = nullptr; }

    // Synchronizes and folds all pending events into stageMs.
    void collectProfile()
    {
        if (pendingEvents.empty()) return;
        ck(cudaStreamSynchronize(stream), "synchronize");
        for (auto& se : pendingEvents)
        {
            int prev = 0;
            for (int k = 1; k < 6; ++k)
            {
                if (!se.used[k]) continue;
                float ms = 0.0f;
                ck(cudaEventElapsedTime(&ms, se.ev[prev], se.ev[k]),
                   "cudaEventElapsedTime");
                stageMs[k - 1] += ms;
                prev = k;
            }
            ++stageRuns;
            freeEvents.push_back(se);
        }
        pendingEvents.clear();
    }

    ~n2p2b_context()
    {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& se : pendingEvents)
            for (auto& e : se.ev) cudaEventDestroy(e);
        for (auto& se : freeEvents)
            for (auto& e : se.ev) cudaEventDestroy(e);
        if (graphExec) cudaGraphExecDestroy(graphExec);
        for (DevBuf* b : {&structOf, &structAtoms, &bsDev, &structEnergy,
                          &revOff, &revEntry, &Ftarget})
            b->release();
        for (DevBuf* b : {&stu.w, &stu.m, &stu.v, &stu.grad, &stu.gpart,
                          &stu.rE,
                          &stu.rF, &stu.u, &stu.loss, &stu.dRange, &stu.list,
                          &stu.listCount})
            b->release();
        for (DevBuf* b : {&sfScale, &nnW, &slotSF, &tcW[0], &tcF[0], &tcW[1],
                          &tcF[1], &ewRange, &ewPerAtom, &posIn, &pos, &elem,
                          &atomsByElem, &cellOf, &cellCount, &cellFill,
                          &cellStart, &cellAtoms, &cellStatus, &nbrCount,
                          &nbrCountElem, &nbrOff, &keyTmp, &key, &nbrIdx,
                          &nbrEl, &dx, &dy, &dz, &dd, &entryAtom, &mirror,
                          &pairF, &dGdr, &G, &dEdG, &dGdrSelf, &Ei, &selfF,
                          &F, &energyOut, &status, &tabGroupsDev,
                          &tabMembersDev})
            b->release();
        if (statusHost) cudaFreeHost(statusHost);
        if (energyHost) cudaFreeHost(energyHost);
        if (ownStream && stream) cudaStreamDestroy(stream);
    }

    // Host-only contexts (device < 0) support setup and potential queries.
    bool hostOnly() const { return device < 0; }

    void activate()
    {
        if (hostOnly())
            throw StateError("ERROR: This context has no CUDA device (it was "
                             "created with device -1 for setup only).\n");
        ck(cudaSetDevice(device), "cudaSetDevice");
    }

    // ---- potential tables ------------------------------------------------

    // Number of (zeta, lambda) shapes if the angular group's members are
    // (eta runs) x shapes -- each run has the same shape list, zeta is
    // integer, rs = 0 -- else 0.  Members are sorted with eta slowest
    // (SymGrpExpAngn::sortMembers), so runs are contiguous.
    static int productShapes(Element const& el, SymGrp const& g)
    {
        std::size_t const M = g.members.size();
        if (M == 0) return 0;
        SymFnc const& f0 = el.sfs[g.members[0]];
        std::size_t ns = 0;
        while (ns < M && el.sfs[g.members[ns]].eta == f0.eta) ++ns;
        if (ns == 0 || ns > 8 || M % ns != 0) return 0;
        for (std::size_t r = 0; r < M / ns; ++r)
        {
            double const eta = el.sfs[g.members[r * ns]].eta;
            if (r > 0 && eta == el.sfs[g.members[(r - 1) * ns]].eta) return 0;
            for (std::size_t s = 0; s < ns; ++s)
            {
                SymFnc const& f = el.sfs[g.members[r * ns + s]];
                SymFnc const& b = el.sfs[g.members[s]];
                if (f.eta != eta || f.rs != 0.0 || !f.useIntegerPow
                    || f.zeta != b.zeta || f.lambda != b.lambda)
                    return 0;
            }
        }
        return (int)ns;
    }

    // Device layout of a potential's networks: per element and layer W
    // (out x in, row-major), W^T and b in one blob (NNParams offsets).
    static void nnBlob(Potential const& pt, NNParams& P,
                       std::vector<double>& blob)
    {
        int const ne = pt.numElements();
        std::memset(&P, 0, sizeof(P));
        P.numElements = ne;
        blob.clear();
        int maxW = 1;
        for (int e = 0; e < ne; ++e)
        {
            NeuralNet const& nn = pt.elements[e].nn;
            if (nn.numLayers > kMaxLayers)
                throw std::runtime_error("ERROR: Too many NN layers.\n");
            P.numLayers[e] = nn.numLayers;
            P.normalizeNeurons = nn.normalizeNeurons ? 1 : 0;
            for (int l = 0; l < nn.numLayers; ++l)
            {
                P.width[e][l] = nn.neurons[l];
                P.act[e][l] = nn.activations[l];
                maxW = std::max(maxW, nn.neurons[l]);
            }
            for (int l = 1; l < nn.numLayers; ++l)
            {
                int const ni = nn.neurons[l - 1], no = nn.neurons[l];
                P.woff[e][l] = (long)blob.size();
                blob.insert(blob.end(), nn.W[l].begin(), nn.W[l].end());
                P.wtoff[e][l] = (long)blob.size();
                for (int j = 0; j < ni; ++j)
                    for (int o = 0; o < no; ++o)
                        blob.push_back(nn.W[l][(std::size_t)o * ni + j]);
                P.boff[e][l] = (long)blob.size();
                blob.insert(blob.end(), nn.b[l].begin(), nn.b[l].end());
            }
        }
        if (maxW > kMaxWidth)
            throw std::runtime_error("ERROR: NN layer wider than supported.\n");
        P.maxWidth = maxW;
    }

    void buildTables()
    {
        sfVariant = -1;
        sfGrid = 0;
        int const ne = pot.numElements();
        if (ne > kMaxElem)
            throw std::runtime_error("ERROR: More elements than the device "
                                     "tables hold.\n");
        maxSF = pot.maxSymmetryFunctions();
        maxSlots = pot.maxSlots();
        if (maxSF > kMaxSF)
            throw std::runtime_error("ERROR: Too many symmetry functions per "
                                     "element for the device tables.\n");
        std::memset(&sfp, 0, sizeof(sfp));
        {
            std::size_t ng = 0, nm = 0;
            for (auto const& el : pot.elements)
            {
                ng += el.groups.size();
                for (auto const& g : el.groups) nm += g.members.size();
            }
            tabGroups.assign(ng, DevGroup{});
            tabMembers.assign(nm, DevMember{});
        }
        sfp.numElements = ne;
        sfp.cutoffType = pot.cutoffType;
        sfp.maxSlots = maxSlots;
        sfp.maxSF = maxSF;
        for (int e = 0; e < ne && e < kMaxElem; ++e)
            sfp.atomicNumber[e] = pot.elements[e].atomicNumber;
        sfp.PI = 4.0 * std::atan(1.0);
        sfp.PI_2 = 2.0 * std::atan(1.0);
        sfp.E = std::exp(1.0);
        sfp.TANH_PRE = std::pow((sfp.E + 1 / sfp.E) / (sfp.E - 1 / sfp.E), 3);
        std::vector<SFScale> scale((std::size_t)ne * maxSF, SFScale{0, 1, 0, 1});
        ewRangeHost.assign((std::size_t)ne * maxSF, Range{0.0, 0.0});
        std::vector<int16_t> slotTab((std::size_t)kMaxElem * kMaxElem
                                     * std::max(maxSlots, 1), (int16_t)-1);
        int gi = 0, mi = 0;
        sfp.maxExp = 1;
        for (int e = 0; e < ne; ++e)
        {
            Element const& el = pot.elements[e];
            sfp.groupBeg[e] = gi;
            int expCount = 0;
            std::vector<std::pair<double, double>> expKeys;
            sfp.numSF[e] = (int)el.sfs.size();
            for (int f = 0; f < ne; ++f)
            {
                sfp.numSlots[e][f] = (int)el.sfTable[f].size();
                for (std::size_t s = 0; s < el.sfTable[f].size(); ++s)
                {
                    slotTab[((std::size_t)e * kMaxElem + f) * maxSlots + s] =
                        (int16_t)el.sfTable[f][s];
                }
            }
            for (auto const& g : el.groups)
            {
                DevGroup& d = tabGroups[gi++];
                d.type = g.type;
                d.e1 = g.e1;
                d.e2 = g.e2;
                d.mbeg = mi;
                d.mcnt = (int)g.members.size();
                d.rc = g.rc;
                d.rc2 = g.rc * g.rc;
                // CutoffFunction::setCutoffRadius / setCutoffParameter.
                d.rcinv = 1.0 / g.rc;
                d.rci = g.rc * g.cutoffAlpha;
                d.iw = 1.0 / (g.rc - d.rci);
                for (std::size_t k = 0; k < g.members.size(); ++k)
                {
                    SymFnc const& s = el.sfs[g.members[k]];
                    DevMember& m = tabMembers[mi++];
                    std::memset(&m, 0, sizeof(m));
                    m.eta = s.eta;
                    m.rs = s.rs;
                    m.lambda = s.lambda;
                    m.zeta = s.zeta;
                    m.zetaInt = (int16_t)s.zetaInt;
                    m.useIntPow = s.useIntegerPow ? 1 : 0;
                    m.rsPositive = s.rs > 0.0 ? 1 : 0;
                    m.sf = (int16_t)s.index;
                    for (int f = 0; f < kMaxElem; ++f)
                        m.slot[f] = (f < ne) ? (int16_t)s.indexPerElement[f]
                                             : (int16_t)-1;
                    SFScale& q = scale[(std::size_t)e * maxSF + s.index];
                    ewRangeHost[(std::size_t)e * maxSF + s.index] =
                        Range{s.Gmin, s.Gmax};
                    if (isCompactType(g.type))
                    {
                        // CompactFunction::setLeftRight
                        // (libnnp/CompactFunction.cpp:60-72) for the radial
                        // and angular functions; angles in radians as
                        // SymFncBaseCompAng::setParameters computes them.
                        m.eta = s.rl;
                        m.rs = s.rc;
                        m.lambda = s.angleLeft * M_PI / 180.0;
                        m.zeta = s.angleRight * M_PI / 180.0;
                        m.factorNorm = s.scalingFactor;
                        m.factorDeriv = (s.rc + s.rl) / 2.0;
                        m.zetaLambda = 1.0 / ((s.rc - s.rl) / 2.0);
                        if (g.type != 20 && g.type != 23)
                        {
                            m.aCenter = (m.lambda + m.zeta) / 2.0;
                            m.aScale = 1.0 / ((m.zeta - m.lambda) / 2.0);
                        }
                        m.zetaInt = (int16_t)s.coreType;
                        m.useIntPow = s.asymmetric ? 1 : 0;
                        // SymGrpCompAngn::sortMembers (calculateComp).
                        SymFnc const* prev = k > 0
                            ? &el.sfs[g.members[k - 1]] : nullptr;
                        m.calcExp = (prev == nullptr || prev->rc != s.rc
                                     || prev->rl != s.rl) ? 1 : 0;
                        // Radial function id: the first member of the group
                        // with the same (rl, rc, core, asymmetry); members
                        // sharing it share their radial values.
                        std::size_t rid = 0;
                        while (rid < k)
                        {
                            SymFnc const& o = el.sfs[g.members[rid]];
                            if (o.rl == s.rl && o.rc == s.rc
                                && o.coreType == s.coreType
                                && o.asymmetric == s.asymmetric)
                                break;
                            ++rid;
                        }
                        m.rsPositive = (uint8_t)rid;
                        q.q = 1.0;
                    }
                    else if (g.type == 2 || g.type == 12)
                    {
                        m.factorNorm = s.scalingFactor;
                        m.calcExp = 1;
                        q.q = 1.0;
                    }
                    else
                    {
                        // SymGrpExpAngn::sortMembers + setScalingFactors.
                        double const fn = std::pow(2.0, 1.0 - s.zeta);
                        m.factorNorm = fn * s.scalingFactor;
                        m.factorDeriv = 2.0 * s.eta / s.zeta / s.lambda;
                        m.zetaLambda = s.zeta * s.lambda;
                        SymFnc const* prev = k > 0
                            ? &el.sfs[g.members[k - 1]] : nullptr;
                        m.calcExp = (prev == nullptr || prev->eta != s.eta
                                     || prev->rs != s.rs) ? 1 : 0;
                        // One exp(-eta (r - rs)^2) table per distinct
                        // (eta, rs) of the element, shared by its groups.
                        int idx = 0;
                        while (idx < (int)expKeys.size()
                               && !(expKeys[idx].first == s.eta
                                    && expKeys[idx].second == s.rs))
                            ++idx;
                        if (idx == (int)expKeys.size())
                        {
                            expKeys.emplace_back(s.eta, s.rs);
                            m.fillExp = 1;
                        }
                        expCount = (int)expKeys.size();
                        m.expIdx = (int16_t)idx;
                        q.q = m.factorNorm / s.scalingFactor;
                    }
                    switch (s.scalingType)
                    {
                    case ST_NONE:        q.smin = 0.0; q.b = 1.0; q.shift = 0.0;
                                         break;
                    case ST_CENTER:      q.smin = 0.0; q.b = 1.0;
                                         q.shift = s.Gmean; break;
                    case ST_SCALE:       q.smin = s.Smin; q.b = s.scalingFactor;
                                         q.shift = s.Gmin; break;
                    default:             q.smin = s.Smin; q.b = s.scalingFactor;
                                         q.shift = s.Gmean; break;
                    }
                }
                d.shapes = (g.type == 2 || g.type == 12 || g.type == 13
                            || isCompactType(g.type))
                         ? 0 : productShapes(el, g);
                // Cosine cutoff without inner radius: for a distance r,
                // f_c = (1 + cos(a r)) / 2 and f_c'(r) / r =
                // -(a^2 / 2) sin(a r) / (a r), a = pi / rc, are power series
                // in v = (a r)^2 = a^2 r^2 (used for r_jk of narrow triplets:
                // no square root; v <= pi^2 there).
                d.cosSeries = (pot.cutoffType == 1 && d.rci == 0.0) ? 1 : 0;
                {
                    double const a = (4.0 * std::atan(1.0)) / g.rc;
                    d.a2 = a * a;
                }
                {
                    int zmax = 0;
                    for (int mi2 : g.members)
                        zmax = std::max(zmax, el.sfs[mi2].zetaInt - 1);
                    int b = 0;
                    while (b < 31 && (zmax >> b) != 0) ++b;
                    d.powBits = b;
                }
            }
            sfp.maxExp = std::max(sfp.maxExp, expCount);
        }
        sfp.groupBeg[ne] = gi;
        sfp.numGroups = gi;
        sfp.numMembers = mi;
        sfp.groups = tabGroups.data();
        sfp.members = tabMembers.data();
        // Tables up to 32 KB are staged in shared memory by the kernels;
        // N2P2B_SF_GLOBAL_TABLES=1 keeps them in global memory (tests).
        {
            std::size_t const b = sizeof(DevGroup) * tabGroups.size()
                                + sizeof(DevMember) * tabMembers.size();
            char const* env = std::getenv("N2P2B_SF_GLOBAL_TABLES");
            sfp.stageTables = (b <= 32 * 1024
                               && !(env && std::atoi(env) != 0)) ? 1 : 0;
        }

        // NN blob.
        std::vector<double> blob;
        nnBlob(pot, nnp, blob);
        std::vector<unsigned char> tcWeights[2];
        std::vector<float> tcFloats[2];
        for (int k = 0; k < 2; ++k)
            tcOk[k] = tcBuild(nnp, blob, k == 1 ? 1 : 2, tcp[k], tcWeights[k],
                              tcFloats[k], tcWhy[k]);

        if (hostOnly())
        {
            tablesReady = true;
            return;
        }
        activate();
        tabGroupsDev.ensure(sizeof(DevGroup) * std::max<std::size_t>(
                                tabGroups.size(), 1));
        tabMembersDev.ensure(sizeof(DevMember) * std::max<std::size_t>(
                                 tabMembers.size(), 1));
        if (!tabGroups.empty())
            ck(cudaMemcpy(tabGroupsDev.p, tabGroups.data(),
                          sizeof(DevGroup) * tabGroups.size(),
                          cudaMemcpyHostToDevice), "copy SF groups");
        if (!tabMembers.empty())
            ck(cudaMemcpy(tabMembersDev.p, tabMembers.data(),
                          sizeof(DevMember) * tabMembers.size(),
                          cudaMemcpyHostToDevice), "copy SF members");
        sfp.dGroups = tabGroupsDev.as<DevGroup>();
        sfp.dMembers = tabMembersDev.as<DevMember>();
        sfScale.ensure(sizeof(SFScale) * scale.size());
        ck(cudaMemcpy(sfScale.p, scale.data(), sizeof(SFScale) * scale.size(),
                      cudaMemcpyHostToDevice), "copy SF scaling");
        sfScaleHost = scale;
        ewRange.ensure(sizeof(Range) * ewRangeHost.size());
        ck(cudaMemcpy(ewRange.p, ewRangeHost.data(),
                      sizeof(Range) * ewRangeHost.size(),
                      cudaMemcpyHostToDevice), "copy SF ranges");
        nnW.ensure(sizeof(double) * blob.size());
        ck(cudaMemcpy(nnW.p, blob.data(), sizeof(double) * blob.size(),
                      cudaMemcpyHostToDevice), "copy NN weights");
        slotSF.ensure(sizeof(int16_t) * slotTab.size());
        ck(cudaMemcpy(slotSF.p, slotTab.data(), sizeof(int16_t) * slotTab.size(),
                      cudaMemcpyHostToDevice), "copy slot table");
        for (int k = 0; k < 2; ++k)
        {
            tcGrid[k] = 0;
            graphValid = false;
            if (!tcOk[k]) continue;
            tcW[k].ensure(tcWeights[k].size());
            ck(cudaMemcpy(tcW[k].p, tcWeights[k].data(), tcWeights[k].size(),
                          cudaMemcpyHostToDevice), "copy BF16 weights");
            tcF[k].ensure(sizeof(float) * tcFloats[k].size());
            ck(cudaMemcpy(tcF[k].p, tcFloats[k].data(),
                          sizeof(float) * tcFloats[k].size(),
                          cudaMemcpyHostToDevice), "copy FP32 NN parameters");
        }
        tablesReady = true;
        invalidate();
    }

    void requireReady() const
    {
        if (!generic || !scaled || !weighted || !tablesReady)
            throw StateError("ERROR: Potential is not set up (settings, "
                             "scaling and weights are required).\n");
    }

    void requireStructure() const
    {
        if (n <= 0) throw StateError("ERROR: No structure set.\n");
    }

    // The network changed: symmetry functions and neighbor list stand.
    void invalidateNN()
    {
        haveNN = haveNNDeriv = haveE = haveF = false;
    }

    void invalidate()
    {
        haveNL = haveSF = haveSFDeriv = haveNN = haveNNDeriv = false;
        haveE = haveF = false;
    }

    // ---- structure -------------------------------------------------------

    // Geometry of one periodic (box != null) or open structure in the
    // units the kernels compute in.
    void structureGeometry(double const* box, double rc, NLParams& q,
                           PhysBox& b, int* cellsOut)
    {
        double const L = pot.normalize ? pot.convLength : 1.0;
        std::memset(&q, 0, sizeof(q));
        std::memset(&b, 0, sizeof(b));
        q.rc2 = rc * rc;
        if (box == nullptr)
        {
            q.periodic = 0;
            q.nimg = 1;
            if (cellsOut) *cellsOut = 0;
            return;
        }
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) b.box[k][c] = box[3 * k + c];
        inverseBox(b.box, b.invbox);
        q.periodic = 1;
        // Structure::toNormalizedUnits: box *= convLength, invbox /= convL.
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c)
            {
                q.box[k][c] = pot.normalize ? b.box[k][c] * L : b.box[k][c];
                q.invbox[k][c] = pot.normalize ? b.invbox[k][c] / L
                                               : b.invbox[k][c];
            }
        double proj[3];
        pbcCopies(q.box, rc, q.pbc, proj);
        q.nimg = (2 * q.pbc[0] + 1) * (2 * q.pbc[1] + 1) * (2 * q.pbc[2] + 1);
        if (!cellsOut) return;
        bool cellOk = true;
        long cells = 1;
        for (int k = 0; k < 3; ++k)
        {
            int nc = (int)std::floor(proj[k] / (rc * (1.0 + 1e-9)));
            nc = std::min(nc, 160);
            if (nc < 1 || q.pbc[k] != 1) cellOk = false;
            q.ncell[k] = nc;
            cells *= std::max(nc, 1);
        }
        if (!cellOk)
        {
            q.ncell[0] = q.ncell[1] = q.ncell[2] = 0;
            *cellsOut = 0;
        }
        else *cellsOut = (int)cells;
    }

    // A batch of independent structures: counts[s] atoms each, boxes
    // (9 doubles per structure) or null for open structures, positions and
    // elements concatenated in structure order.
    void setStructures(long num, int64_t const* counts, double const* boxes,
                       double const* posArg, int loc, int32_t const* elems,
                       int flags)
    {
        requireReady();
        if (num <= 0 || !counts || !posArg || !elems)
            throw std::invalid_argument("ERROR: Invalid batch arguments.\n");
        long total = 0;
        for (long s = 0; s < num; ++s)
        {
            if (counts[s] <= 0)
                throw std::invalid_argument("ERROR: Empty structure in "
                                            "batch.\n");
            total += counts[s];
        }
        if (total > 0x7ffffffeL / 2)
            throw std::invalid_argument("ERROR: Too many atoms.\n");
        int const ne = pot.numElements();
        for (long i = 0; i < total; ++i)
            if (elems[i] < 0 || elems[i] >= ne)
                throw std::invalid_argument("ERROR: Element index out of "
                                            "range.\n");
        activate();
        n = total;
        numStructs = num;
        externalNL = false;
        sfCap = 0;
        lastMaxNbr = 0;
        elemHost.assign(elems, elems + total);
        periodic = boxes != nullptr;
        remap = periodic && (flags & N2P2B_REMAP);
        numCells = 0;
        std::memset(&nlp, 0, sizeof(nlp));
        std::memset(&pb, 0, sizeof(pb));
        double const rc = pot.maxCutoffRadius;
        bsHost.assign(num, BatchStruct{});
        structCounts.assign(counts, counts + num);
        std::vector<int> sOf(total), sAtoms(total);
        batchNIMG = 1;
        long a0 = 0;
        for (long s = 0; s < num; ++s)
        {
            BatchStruct& B = bsHost[s];
            structureGeometry(boxes ? boxes + 9 * s : nullptr, rc, B.p, B.pb,
                              nullptr);
            B.doRemap = remap ? 1 : 0;
            B.atomBeg = (int)a0;
            B.atomEnd = (int)(a0 + counts[s]);
            int k = (int)a0;
            for (int e = 0; e < ne; ++e)
            {
                B.es[e] = k;
                for (long i = a0; i < a0 + counts[s]; ++i)
                    if (elemHost[i] == e) sAtoms[k++] = (int)i;
            }
            for (int e = ne; e <= kMaxElem; ++e) B.es[e] = k;
            for (long i = a0; i < a0 + counts[s]; ++i) sOf[i] = (int)s;
            batchNIMG = std::max(batchNIMG, B.p.nimg);
            a0 += counts[s];
        }
        if ((long double)n * batchNIMG * kMaxElem > 1.8e19L)
            throw std::invalid_argument("ERROR: Batch too large for the "
                                        "neighbor keys.\n");
        nlp.nimg = batchNIMG;
        // Element-sorted atoms of the whole batch (tensor-core tiles,
        // training blocks).
        std::vector<int> byElem;
        byElem.reserve(n);
        std::memset(&es, 0, sizeof(es));
        for (int e = 0; e < ne; ++e)
        {
            es.start[e] = (int)byElem.size();
            for (long i = 0; i < n; ++i)
                if (elemHost[i] == e) byElem.push_back((int)i);
        }
        es.start[ne] = (int)byElem.size();
        for (int e = ne + 1; e <= kMaxElem; ++e) es.start[e] = es.start[ne];
        posIn.ensure(sizeof(double) * 3 * n);
        pos.ensure(sizeof(double) * 3 * n);
        elem.ensure(sizeof(int) * n);
        atomsByElem.ensure(sizeof(int) * n);
        structOf.ensure(sizeof(int) * n);
        structAtoms.ensure(sizeof(int) * n);
        bsDev.ensure(sizeof(BatchStruct) * num);
        structEnergy.ensure(sizeof(double) * num);
        ck(cudaMemcpyAsync(elem.p, elemHost.data(), sizeof(int) * n,
                           cudaMemcpyHostToDevice, stream), "copy elements");
        ck(cudaMemcpyAsync(atomsByElem.p, byElem.data(), sizeof(int) * n,
                           cudaMemcpyHostToDevice, stream), "copy atom lists");
        ck(cudaMemcpyAsync(structOf.p, sOf.data(), sizeof(int) * n,
                           cudaMemcpyHostToDevice, stream), "copy batch map");
        ck(cudaMemcpyAsync(structAtoms.p, sAtoms.data(), sizeof(int) * n,
                           cudaMemcpyHostToDevice, stream), "copy batch lists");
        ck(cudaMemcpyAsync(bsDev.p, bsHost.data(), sizeof(BatchStruct) * num,
                           cudaMemcpyHostToDevice, stream), "copy batch");
        setPositions(posArg, loc);
        ck(cudaStreamSynchronize(stream), "batch upload");
        graphValid = false;
        applyTuned();
    }

    void setStructure(long num, double const* box, double const* posArg,
                      int loc, int32_t const* elems, int flags)
    {
        numStructs = 0;
        externalNL = false;
        graphValid = false;
        requireReady();
        if (num <= 0 || posArg == nullptr || elems == nullptr)
            throw std::invalid_argument("ERROR: Invalid structure "
                                        "arguments.\n");
        if (num > 0x7ffffffeL / 2)
            throw std::invalid_argument("ERROR: Too many atoms.\n");
        int const ne = pot.numElements();
        for (long i = 0; i < num; ++i)
        {
            if (elems[i] < 0 || elems[i] >= ne)
                throw std::invalid_argument("ERROR: Element index out of "
                                            "range.\n");
        }
        activate();
        n = num;
        sfCap = 0;
        lastMaxNbr = 0;
        elemHost.assign(elems, elems + num);
        periodic = box != nullptr;
        remap = periodic && (flags & N2P2B_REMAP);
        double const L = pot.normalize ? pot.convLength : 1.0;
        std::memset(&nlp, 0, sizeof(nlp));
        std::memset(&pb, 0, sizeof(pb));
        double const rc = pot.maxCutoffRadius;
        nlp.rc2 = rc * rc;
        if (periodic)
        {
            for (int k = 0; k < 3; ++k)
                for (int c = 0; c < 3; ++c) boxPhys[k][c] = box[3 * k + c];
            std::memcpy(pb.box, boxPhys, sizeof(boxPhys));
            inverseBox(pb.box, pb.invbox);
            nlp.periodic = 1;
            // Structure::toNormalizedUnits: box *= convLength,
            // invbox /= convLength.
            for (int k = 0; k < 3; ++k)
            {
                for (int c = 0; c < 3; ++c)
                {
                    nlp.box[k][c] = pot.normalize ? pb.box[k][c] * L
                                                  : pb.box[k][c];
                    nlp.invbox[k][c] = pot.normalize ? pb.invbox[k][c] / L
                                                     : pb.invbox[k][c];
                }
            }
            double proj[3];
            pbcCopies(nlp.box, rc, nlp.pbc, proj);
            nlp.nimg = (2 * nlp.pbc[0] + 1) * (2 * nlp.pbc[1] + 1)
                     * (2 * nlp.pbc[2] + 1);
            bool cellOk = true;
            long cells = 1;
            for (int k = 0; k < 3; ++k)
            {
                int nc = (int)std::floor(proj[k] / (rc * (1.0 + 1e-9)));
                nc = std::min(nc, 160);
                if (nc < 1 || nlp.pbc[k] != 1) cellOk = false;
                nlp.ncell[k] = nc;
                cells *= std::max(nc, 1);
            }
            if (!cellOk)
            {
                nlp.ncell[0] = nlp.ncell[1] = nlp.ncell[2] = 0;
                numCells = 0;
            }
            else numCells = (int)cells;
        }
        else
        {
            nlp.periodic = 0;
            nlp.nimg = 1;
            numCells = 0;
        }
        if ((long double)n * nlp.nimg * kMaxElem > 1.8e19L)
            throw std::invalid_argument("ERROR: Structure too large for the "
                                        "neighbor keys.\n");
        // Element-sorted atom lists (brute-force enumeration order).
        std::vector<int> byElem;
        byElem.reserve(n);
        std::memset(&es, 0, sizeof(es));
        for (int e = 0; e < ne; ++e)
        {
            es.start[e] = (int)byElem.size();
            for (long i = 0; i < n; ++i)
                if (elemHost[i] == e) byElem.push_back((int)i);
        }
        es.start[ne] = (int)byElem.size();
        for (int e = ne + 1; e <= kMaxElem; ++e) es.start[e] = es.start[ne];

        posIn.ensure(sizeof(double) * 3 * n);
        pos.ensure(sizeof(double) * 3 * n);
        elem.ensure(sizeof(int) * n);
        atomsByElem.ensure(sizeof(int) * n);
        ck(cudaMemcpyAsync(elem.p, elemHost.data(), sizeof(int) * n,
                           cudaMemcpyHostToDevice, stream), "copy elements");
        ck(cudaMemcpyAsync(atomsByElem.p, byElem.data(), sizeof(int) * n,
                           cudaMemcpyHostToDevice, stream), "copy atom lists");
        setPositions(posArg, loc);
        ck(cudaStreamSynchronize(stream), "structure upload");
        applyTuned();
    }

    void setPositions(double const* posArg, int loc)
    {
        requireStructure();
        ck(cudaMemcpyAsync(posIn.p, posArg, sizeof(double) * 3 * n,
                           loc == N2P2B_DEVICE ? cudaMemcpyDeviceToDevice
                                               : cudaMemcpyHostToDevice,
                           stream), "copy positions");
        invalidate();
    }

    // ---- buffers ---------------------------------------------------------

    void ensureStructureBuffers()
    {
        int const ne = pot.numElements();
        cellOf.ensure(sizeof(int) * n);
        cellAtoms.ensure(sizeof(int) * n);
        cellCount.ensure(sizeof(int) * (numCells + 1));
        cellFill.ensure(sizeof(int) * (numCells + 1));
        cellStart.ensure(sizeof(int) * (numCells + 1));
        cellStatus.ensure(sizeof(int) * ST_NUM);
        nbrCount.ensure(sizeof(int) * n);
        nbrCountElem.ensure(sizeof(int) * n * ne);
        nbrOff.ensure(sizeof(int) * (n + 1));
        G.ensure(realBytes() * n * maxSF);
        dEdG.ensure(realBytes() * n * maxSF);
        Ei.ensure(sizeof(double) * n);
        ewPerAtom.ensure(sizeof(int) * n);
        if (stu.loaded) stu.list.ensure(sizeof(int) * n);
        selfF.ensure(sizeof(double) * n * 3);
        F.ensure(sizeof(double) * n * 3);
        energyOut.ensure(sizeof(double) * 2);
        status.ensure(sizeof(int) * ST_NUM);
        if (!statusHost)
            ck(cudaMallocHost((void**)&statusHost, sizeof(int) * ST_NUM),
               "cudaMallocHost");
        if (!energyHost)
            ck(cudaMallocHost((void**)&energyHost, sizeof(double) * 2),
               "cudaMallocHost");
    }

    void ensureEntryBuffers()
    {
        long const c = std::max(capacity, 1L);
        keyTmp.ensure(sizeof(unsigned long long) * c);
        key.ensure(sizeof(unsigned long long) * c);
        nbrIdx.ensure(sizeof(int) * c);
        nbrEl.ensure(sizeof(int8_t) * c);
        dx.ensure(sizeof(double) * c);
        dy.ensure(sizeof(double) * c);
        dz.ensure(sizeof(double) * c);
        dd.ensure(sizeof(double) * c);
        entryAtom.ensure(sizeof(int) * c);
        mirror.ensure(sizeof(int) * c);
        pairF.ensure(sizeof(double) * 3 * c);
        dGdr.ensure(realBytes() * 3 * (std::size_t)c
                    * std::max(maxSlots, 1));
    }

    // Bytes of one symmetry-function / dE/dG / dG/dr value.
    std::size_t realBytes() const
    {
        return precision != PREC_FP64 ? sizeof(float) : sizeof(double);
    }

    // Copies `count` values of a per-atom real buffer to the host as double.
    std::vector<double> readReal(DevBuf const& b, std::size_t count)
    {
        std::vector<double> out(count);
        if (count == 0) return out;
        if (precision != PREC_FP64)
        {
            std::vector<float> f(count);
            ck(cudaMemcpy(f.data(), b.p, sizeof(float) * count,
                          cudaMemcpyDeviceToHost), "read results");
            for (std::size_t k = 0; k < count; ++k) out[k] = f[k];
        }
        else
        {
            ck(cudaMemcpy(out.data(), b.p, sizeof(double) * count,
                          cudaMemcpyDeviceToHost), "read results");
        }
        return out;
    }

    void setPrecision(int mode)
    {
        if (mode != PREC_FP64 && mode != PREC_MIXED && mode != PREC_BF16)
            throw std::invalid_argument("ERROR: Unknown precision mode.\n");
        int const k = (mode == PREC_MIXED) ? 1 : 0;
        if (mode != PREC_FP64 && tablesReady && !tcOk[k])
            throw std::runtime_error("ERROR: The mixed-precision form cannot "
                                     "run this potential: " + tcWhy[k]
                                     + ".\n");
        if (mode == precision) return;
        precision = mode;
        sfGrid = 0;
        graphValid = false;
        invalidate();
        applyTuned();
        if (n > 0 && !hostOnly())
        {
            activate();
            ensureStructureBuffers();
            ensureEntryBuffers();
        }
    }

    void grow(long total)
    {
        // Batches hold tens of millions of entries: keep the headroom small.
        double const headroom = numStructs > 0 ? 1.02 : 1.15;
        capacity = std::max(capacity, (long)(total * headroom) + 1024);
        graphValid = false;
        ensureEntryBuffers();
    }

    // ---- pipeline stages (enqueue only) -----------------------------------

    void enqueueReset()
    {
        noteLaunches(2);
        statusResetKernel<<<1, 32, 0, stream>>>(status.as<int>());
        statusResetKernel<<<1, 32, 0, stream>>>(cellStatus.as<int>());
    }

    void enqueueNL()
    {
        if (externalNL) return;      // the caller's list is already in place
        if (numStructs > 0)
        {
            NLBatchLaunch B;
            B.n = (int)n;
            B.numElements = pot.numElements();
            B.NIMG = batchNIMG;
            B.capacity = capacity;
            B.warpsPerBlock = nlWarpsPerBlock;
            B.normalize = pot.normalize ? 1 : 0;
            B.convLength = pot.convLength;
            B.bs = bsDev.as<BatchStruct>();
            B.structOf = structOf.as<int>();
            B.structAtoms = structAtoms.as<int>();
            B.posIn = posIn.as<double>();
            B.pos = pos.as<double>();
            B.elem = elem.as<int>();
            B.nbrCount = nbrCount.as<int>();
            B.nbrCountElem = nbrCountElem.as<int>();
            B.nbrOff = nbrOff.as<int>();
            B.key = key.as<unsigned long long>();
            B.nbrIdx = nbrIdx.as<int>();
            B.nbrEl = nbrEl.as<int8_t>();
            B.dx = dx.as<double>();
            B.dy = dy.as<double>();
            B.dz = dz.as<double>();
            B.dd = dd.as<double>();
            B.entryAtom = entryAtom.as<int>();
            B.mirror = mirror.as<int>();
            B.status = status.as<int>();
            launchNeighborListBatch(B, stream);
            return;
        }
        NLLaunch L;
        L.n = (int)n;
        L.numElements = pot.numElements();
        L.numCells = numCells;
        L.capacity = capacity;
        L.p = nlp;
        L.pb = pb;
        L.doRemap = remap ? 1 : 0;
        L.normalize = pot.normalize ? 1 : 0;
        L.convLength = pot.convLength;
        L.posIn = posIn.as<double>();
        L.pos = pos.as<double>();
        L.elem = elem.as<int>();
        L.atomsByElem = atomsByElem.as<int>();
        L.es = es;
        L.cellOf = cellOf.as<int>();
        L.cellCount = cellCount.as<int>();
        L.cellStart = cellStart.as<int>();
        L.cellFill = cellFill.as<int>();
        L.cellAtoms = cellAtoms.as<int>();
        L.cellScanStatus = cellStatus.as<int>();
        L.nbrCount = nbrCount.as<int>();
        L.nbrCountElem = nbrCountElem.as<int>();
        L.nbrOff = nbrOff.as<int>();
        L.keyTmp = keyTmp.as<unsigned long long>();
        L.key = key.as<unsigned long long>();
        L.nbrIdx = nbrIdx.as<int>();
        L.nbrEl = nbrEl.as<int8_t>();
        L.dx = dx.as<double>();
        L.dy = dy.as<double>();
        L.dz = dz.as<double>();
        L.dd = dd.as<double>();
        L.entryAtom = entryAtom.as<int>();
        L.mirror = mirror.as<int>();
        L.status = status.as<int>();
        launchNeighborList(L, stream);
    }

    void enqueueSF(bool deriv)
    {
        if (sfVariant < 0)
        {
            sfVariant = sfDefaultVariant(sfp, precision);
            if (char const* v = std::getenv("N2P2B_SF_VARIANT"))
                sfVariant = std::atoi(v);
            sfSortCats = sfDefaultSort(sfp);
            if (char const* v = std::getenv("N2P2B_SF_SORT"))
                sfSortCats = std::atoi(v);
        }
        if (sfGrid == 0 || sfGridCap != sfCap)
        {
            ck(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount,
                                      device), "device attribute");
            sfGrid = smCount * sfBlocksPerSM(sfp, sfCap, sfVariant, precision);
            sfGridCap = sfCap;
        }
        int const perBlock = sfAtomsPerBlock(sfp, sfVariant);
        long const blocksNeeded = (n + perBlock - 1) / perBlock;
        SFLaunch L;
        L.n = (int)n;
        L.derivatives = deriv ? 1 : 0;
        L.cap = sfCap;
        L.memberChunk = 12;
        L.grid = (int)std::max<long>(1, std::min<long>(sfGrid, blocksNeeded));
        L.variant = sfVariant;
        L.sortCats = sfSortCats;
        L.elem = elem.as<int>();
        L.nbrOff = nbrOff.as<int>();
        L.nbrCountElem = nbrCountElem.as<int>();
        L.dx = dx.as<double>();
        L.dy = dy.as<double>();
        L.dz = dz.as<double>();
        L.dd = dd.as<double>();
        L.scale = sfScale.as<SFScale>();
        L.precision = precision;
        L.G = G.p;
        L.dGdr = dGdr.p;
        L.status = status.as<int>();
        launchSymmetryFunctions(sfp, L, stream);
    }

    // Element::updateSymmetryFunctionStatistics for every atom.
    void enqueueEW()
    {
        EWLaunch L;
        L.n = (int)n;
        L.maxSF = maxSF;
        L.precision = precision;
        for (int e = 0; e < pot.numElements(); ++e) L.numSF[e] = sfp.numSF[e];
        L.elem = elem.as<int>();
        L.G = G.p;
        L.scale = sfScale.as<SFScale>();
        L.range = ewRange.as<Range>();
        L.perAtom = ewPerAtom.as<int>();
        L.status = status.as<int>();
        launchExtrapolationCheck(L, stream);
    }

    // Accounts the warnings of a finished evaluation (status words read).
    void accountEW()
    {
        int const cnt = statusHost[ST_EW_COUNT];
        haveEW = true;
        ewTotal += cnt;
        if (cnt <= 0) return;
        std::string first;
        if (ewWrite || ewStop) first = ewLines(ewWrite);
        if (ewStop)
            throw ExtrapolationError(first + "ERROR: Symmetry function value "
                                     "out of range.\n");
    }

    // The warnings of the last evaluation as the reference records them
    // (Element::updateSymmetryFunctionStatistics, Element.cpp:462-541, atom
    // by atom, each atom's symmetry functions in order): the unscaled value
    // (SymFnc::unscale of the kernel's G) outside [Gmin, Gmax] by more than
    // 1000 DBL_EPSILON.
    std::vector<n2p2b_extrapolation_warning> ewRecords()
    {
        std::vector<n2p2b_extrapolation_warning> out;
        std::vector<int> per(n);
        ck(cudaMemcpy(per.data(), ewPerAtom.p, sizeof(int) * n,
                      cudaMemcpyDeviceToHost), "read warnings");
        std::vector<double> const g = readReal(G, (std::size_t)n * maxSF);
        double const eps = 1000.0 * DBL_EPSILON;
        for (long i = 0; i < n; ++i)
        {
            if (per[i] == 0) continue;
            int const e = elemHost[i];
            Element const& el = pot.elements[e];
            for (std::size_t s = 0; s < el.sfs.size(); ++s)
            {
                SFScale const& q = sfScaleHost[(std::size_t)e * maxSF + s];
                Range const& r = ewRangeHost[(std::size_t)e * maxSF + s];
                double const v = (g[(std::size_t)i * maxSF + s] - q.smin) / q.b
                               + q.shift;
                if (!(v + eps < r.lo || v - eps > r.hi)) continue;
                n2p2b_extrapolation_warning w{};
                w.atom = i;
                w.element = e;
                w.sf = (int32_t)s;
                w.type = el.sfs[s].type;
                w.value = v;
                w.gmin = r.lo;
                w.gmax = r.hi;
                out.push_back(w);
            }
        }
        return out;
    }

    // The reference's warning lines (Element.cpp:505-518) for the last
    // evaluation; prints all of them when `print`, returns the first.
    std::string ewLines(bool print)
    {
        std::string first;
        for (n2p2b_extrapolation_warning const& w : ewRecords())
        {
            Element const& el = pot.elements[w.element];
            char buf[256];
            std::snprintf(buf, sizeof(buf),
                          "### NNP EXTRAPOLATION WARNING ### STRUCTURE: "
                          "%6zu ATOM: %9ld ELEMENT: %2s SYMFUNC: %4zu "
                          "TYPE: %2d VALUE: %10.3E MIN: %10.3E MAX: "
                          "%10.3E\n", (std::size_t)0, (long)w.atom,
                          el.symbol.c_str(), (std::size_t)w.sf + 1, w.type,
                          w.value, w.gmin, w.gmax);
            if (first.empty()) first = buf;
            if (print) std::fputs(buf, stderr);
        }
        return first;
    }

    // ---- distilled student ------------------------------------------------

    static bool sameSF(SymFnc const& a, SymFnc const& b)
    {
        return a.type == b.type && a.ec == b.ec && a.e1 == b.e1
            && a.e2 == b.e2 && a.eta == b.eta && a.rs == b.rs && a.rc == b.rc
            && a.zeta == b.zeta && a.lambda == b.lambda && a.rl == b.rl
            && a.angleLeft == b.angleLeft && a.angleRight == b.angleRight
            && a.subtype == b.subtype
            && a.cutoffType == b.cutoffType && a.cutoffAlpha == b.cutoffAlpha
            && a.scalingType == b.scalingType && a.Smin == b.Smin
            && a.Smax == b.Smax && a.Gmin == b.Gmin && a.Gmax == b.Gmax
            && a.Gmean == b.Gmean && a.Gsigma == b.Gsigma;
    }

    // Loads a student potential directory: input.nn with this potential's
    // symmetry functions, its scaling.data, the student's
    // weights.%03zu.data and (once trained) training_range.data.
    void setupStudent(std::string d)
    {
        requireReady();
        if (!d.empty() && d.back() != '/') d += "/";
        Student s;
        s.pot.loadSettingsFile(d + "input.nn");
        s.pot.setupGeneric();
        s.pot.setupSymmetryFunctionScaling(d + "scaling.data");
        s.pot.setupNeuralNetworkWeights(d + "weights.%03zu.data");
        int const ne = pot.numElements();
        if (s.pot.numElements() != ne)
            throw std::runtime_error("ERROR: The student has other elements "
                                     "than the potential.\n");
        for (int e = 0; e < ne; ++e)
        {
            Element const& a = pot.elements[e];
            Element const& b = s.pot.elements[e];
            if (a.symbol != b.symbol || a.sfs.size() != b.sfs.size())
                throw std::runtime_error("ERROR: The student's elements or "
                                         "symmetry functions differ from the "
                                         "potential's.\n");
            for (std::size_t k = 0; k < a.sfs.size(); ++k)
                if (!sameSF(a.sfs[k], b.sfs[k]))
                    throw std::runtime_error(
                        "ERROR: The student's symmetry functions or scaling "
                        "differ from the potential's.\n");
        }
        std::vector<double> bd;
        nnBlob(s.pot, s.nnp, bd);
        s.blob.assign(bd.begin(), bd.end());
        s.trainable = true;
        for (int e = 0; e < ne; ++e)
        {
            NNParams const& q = s.nnp;
            bool const ok = q.numLayers[e] == 3 && q.act[e][1] == AF_TANH
                         && q.act[e][2] == AF_IDENTITY && q.width[e][2] == 1
                         && !q.normalizeNeurons && q.width[e][1] <= 64;
            if (!ok)
            {
                s.trainable = false;
                s.whyNot = "training needs one hidden tanh layer (<= 64 "
                           "neurons), a linear single output and no "
                           "normalize_nodes";
            }
            s.maxH = std::max(s.maxH, q.width[e][1]);
            s.maxNin = std::max(s.maxNin, q.width[e][0]);
            s.maxParams = std::max(s.maxParams, q.width[e][1] * q.width[e][0]
                                                + 2 * q.width[e][1] + 1);
        }
        s.range.assign((std::size_t)ne * maxSF, Range{DBL_MAX, -DBL_MAX});
        std::ifstream rf(d + "training_range.data");
        if (rf.is_open())
        {
            std::string line;
            while (std::getline(rf, line))
            {
                if (line.empty() || line[0] == '#') continue;
                std::istringstream is(line);
                int e = 0, k = 0;
                double lo = 0.0, hi = 0.0;
                if (!(is >> e >> k >> lo >> hi)) continue;
                if (e < 1 || e > ne || k < 1 || k > maxSF)
                    throw std::runtime_error("ERROR: Bad training_range.data "
                                             "line.\n");
                s.range[(std::size_t)(e - 1) * maxSF + (k - 1)] =
                    Range{lo, hi};
            }
            s.haveRange = true;
        }
        s.loaded = true;
        // Keep the device buffers of a previous student (grow-only).
        std::swap(s.w, stu.w);
        std::swap(s.m, stu.m);
        std::swap(s.v, stu.v);
        std::swap(s.grad, stu.grad);
        std::swap(s.gpart, stu.gpart);
        std::swap(s.rE, stu.rE);
        std::swap(s.rF, stu.rF);
        std::swap(s.u, stu.u);
        std::swap(s.loss, stu.loss);
        std::swap(s.dRange, stu.dRange);
        std::swap(s.list, stu.list);
        std::swap(s.listCount, stu.listCount);
        std::swap(s.lrScale, stu.lrScale);
        stu = std::move(s);
        if (hostOnly()) return;
        activate();
        stu.w.ensure(sizeof(float) * stu.blob.size());
        ck(cudaMemcpy(stu.w.p, stu.blob.data(), sizeof(float) * stu.blob.size(),
                      cudaMemcpyHostToDevice), "copy student weights");
        resetOptimizer();
        stu.dRange.ensure(sizeof(Range) * stu.range.size());
        ck(cudaMemcpy(stu.dRange.p, stu.range.data(),
                      sizeof(Range) * stu.range.size(),
                      cudaMemcpyHostToDevice), "copy training range");
        // Adam's W1 learning-rate factors: 1 / sigma of each input
        // (scaling.data), sigma floored at 1e-3 of the element's largest.
        {
            std::vector<float> lrs((std::size_t)ne * maxSF, 1.0f);
            for (int e = 0; e < ne; ++e)
            {
                auto const& sfs = stu.pot.elements[e].sfs;
                double smax = 0.0;
                for (auto const& f : sfs) smax = std::max(smax, f.Gsigma);
                if (!(smax > 0.0)) continue;
                for (auto const& f : sfs)
                    lrs[(std::size_t)e * maxSF + f.index] =
                        (float)(1.0 / std::max(f.Gsigma, 1e-3 * smax));
            }
            stu.lrScale.ensure(sizeof(float) * lrs.size());
            ck(cudaMemcpy(stu.lrScale.p, lrs.data(), sizeof(float) * lrs.size(),
                          cudaMemcpyHostToDevice), "copy learning rates");
        }
        stu.listCount.ensure(sizeof(int) * kMaxElem);
        stu.loss.ensure(sizeof(double) * 2);
        if (n > 0) stu.list.ensure(sizeof(int) * n);
        invalidate();
    }

    void resetOptimizer()
    {
        stu.m.ensure(sizeof(float) * stu.blob.size());
        stu.v.ensure(sizeof(float) * stu.blob.size());
        stu.grad.ensure(sizeof(float) * stu.blob.size());
        ck(cudaMemsetAsync(stu.grad.p, 0, sizeof(float) * stu.blob.size(),
                           stream), "clear gradient");
        ck(cudaMemsetAsync(stu.m.p, 0, sizeof(float) * stu.blob.size(), stream),
           "clear Adam state");
        ck(cudaMemsetAsync(stu.v.p, 0, sizeof(float) * stu.blob.size(), stream),
           "clear Adam state");
        stu.step = 0;
    }

    void requireStudent(bool train) const
    {
        if (!stu.loaded)
            throw StateError("ERROR: No student network set up.\n");
        if (train && !stu.trainable)
            throw std::runtime_error("ERROR: The student cannot be trained: "
                                     + stu.whyNot + ".\n");
        if (precision == PREC_FP64)
            throw StateError("ERROR: The student runs on FP32 symmetry "
                             "functions: select a mixed precision first.\n");
    }

    void setStudentMode(int mode)
    {
        if (mode < 0 || mode > 2)
            throw std::invalid_argument("ERROR: Unknown student mode.\n");
        if (mode != 0)
        {
            requireStudent(false);
            if (mode == 1 && !stu.haveRange)
                throw StateError("ERROR: The gated student needs its "
                                 "training range.\n");
            if (mode == 1 && !tcOk[precision == PREC_MIXED ? 1 : 0])
                throw std::runtime_error("ERROR: The gated student needs the "
                                         "tensor-core form of the potential: "
                                         + tcWhy[precision == PREC_MIXED]
                                         + ".\n");
        }
        stu.mode = mode;
        graphValid = false;
        invalidateNN();
    }

    void enqueueStudentNN(bool deriv)
    {
        NNLaunch L;
        L.n = (int)n;
        L.derivatives = deriv ? 1 : 0;
        L.maxSF = maxSF;
        L.precision = PREC_MIXED;
        L.elem = elem.as<int>();
        L.weights = stu.w.p;
        L.G = G.p;
        L.energy = Ei.as<double>();
        L.dEdG = dEdG.p;
        L.status = status.as<int>();
        launchNeuralNetworks(stu.nnp, L, stream);
    }

    // Student for every atom; atoms with any symmetry function outside the
    // student's training range are re-evaluated by the potential's own
    // network on the tensor cores.
    void enqueueGatedStudent(bool deriv)
    {
        enqueueStudentNN(deriv);
        if (stu.mode != 1) return;
        int const k = (precision == PREC_MIXED) ? 1 : 0;
        ck(cudaMemsetAsync(stu.listCount.p, 0, sizeof(int) * kMaxElem, stream),
           "clear gate lists");
        EWLaunch E;
        E.n = (int)n;
        E.maxSF = maxSF;
        E.precision = precision;
        for (int e = 0; e < pot.numElements(); ++e)
        {
            E.numSF[e] = sfp.numSF[e];
            E.listStart[e] = es.start[e];
        }
        E.elem = elem.as<int>();
        E.G = G.p;
        E.scale = sfScale.as<SFScale>();
        E.range = stu.dRange.as<Range>();
        E.list = stu.list.as<int>();
        E.listCount = stu.listCount.as<int>();
        E.status = status.as<int>();
        E.countSlot = ST_GATE_COUNT;
        launchExtrapolationCheck(E, stream);
        if (tcGrid[k] == 0)
        {
            ck(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount,
                                      device), "device attribute");
            tcGrid[k] = smCount * tcBlocksPerSM(tcp[k]);
        }
        TcNNLaunch T;
        T.n = (int)n;
        T.derivatives = deriv ? 1 : 0;
        T.maxSF = maxSF;
        T.atomsByElem = stu.list.as<int>();
        T.es = es;
        T.listCount = stu.listCount.as<int>();
        T.grid = tcGrid[k];
        T.wblob = tcW[k].as<unsigned char>();
        T.fblob = tcF[k].as<float>();
        T.G = G.as<float>();
        T.energy = Ei.as<double>();
        T.dEdG = dEdG.as<float>();
        T.status = status.as<int>();
        launchNeuralNetworksTC(tcp[k], T, stream);
    }

    long gatedCount()
    {
        requireStudent(false);
        if (stu.mode != 1) return 0;
        int c[kMaxElem] = {};
        ck(cudaMemcpy(c, stu.listCount.p, sizeof(int) * kMaxElem,
                      cudaMemcpyDeviceToHost), "read gate counts");
        long t = 0;
        for (int e = 0; e < pot.numElements(); ++e) t += c[e];
        return t;
    }

    // One Adam step of the student on a batch of the current structure's
    // atoms (symmetry functions and derivatives must be current).
    void studentTrainStep(double const* labelE, double const* labelF,
                          int const* batch, int batchSize, double wE,
                          double wF, double lr, double* lossOut)
    {
        requireStudent(true);
        if (!haveSF || !haveSFDeriv)
            throw StateError("ERROR: Calculate the symmetry functions with "
                             "derivatives first.\n");
        if (batchSize <= 0 || !labelE || !labelF || !batch)
            throw std::invalid_argument("ERROR: Bad training batch.\n");
        activate();
        enqueueStudentNN(true);
        enqueueForces();
        stu.rE.ensure(sizeof(float) * n);
        stu.rF.ensure(sizeof(float) * n * 3);
        stu.u.ensure(sizeof(float) * n * maxSF);
        ck(cudaMemsetAsync(stu.rE.p, 0, sizeof(float) * n, stream), "memset");
        ck(cudaMemsetAsync(stu.rF.p, 0, sizeof(float) * n * 3, stream),
           "memset");
        ck(cudaMemsetAsync(stu.loss.p, 0, sizeof(double) * 2, stream),
           "memset");
        StudentLaunch S;
        int const ne = pot.numElements();
        S.n = (int)n;
        S.maxSF = maxSF;
        S.maxSlots = maxSlots;
        S.numElements = ne;
        S.precision = precision;
        for (int e = 0; e < ne; ++e)
        {
            S.numSF[e] = sfp.numSF[e];
            for (int f = 0; f < ne; ++f) S.numSlots[e][f] = sfp.numSlots[e][f];
            S.hidden[e] = stu.nnp.width[e][1];
            S.woff1[e] = stu.nnp.woff[e][1];
            S.wtoff1[e] = stu.nnp.wtoff[e][1];
            S.boff1[e] = stu.nnp.boff[e][1];
            S.woff2[e] = stu.nnp.woff[e][2];
            S.wtoff2[e] = stu.nnp.wtoff[e][2];
            S.boff2[e] = stu.nnp.boff[e][2];
        }
        S.elem = elem.as<int>();
        S.nbrOff = nbrOff.as<int>();
        S.nbrIdx = nbrIdx.as<int>();
        S.nbrCountElem = nbrCountElem.as<int>();
        S.slotSF = slotSF.as<int16_t>();
        S.atomsByElem = atomsByElem.as<int>();
        S.es = es;
        int const blocks = studentGradBlocks(es, ne, S.blkBeg);
        S.paramStride = stu.maxParams;
        stu.gpart.ensure(sizeof(float) * std::max(blocks, 1)
                         * (std::size_t)stu.maxParams);
        S.G = G.p;
        S.dGdr = dGdr.p;
        S.Ei = Ei.as<double>();
        S.F = F.as<double>();
        S.labelE = labelE;
        S.labelF = labelF;
        S.batch = batch;
        S.batchSize = batchSize;
        S.wE = wE;
        S.wF = wF;
        S.eScale = pot.normalize ? 1.0 / pot.convEnergy : 1.0;
        S.fScale = pot.normalize ? pot.convLength / pot.convEnergy : 1.0;
        S.rE = stu.rE.as<float>();
        S.rF = stu.rF.as<float>();
        S.u = stu.u.as<float>();
        S.blob = stu.w.as<float>();
        S.m = stu.m.as<float>();
        S.v = stu.v.as<float>();
        S.gpart = stu.gpart.as<float>();
        S.grad = stu.grad.as<float>();
        S.loss = stu.loss.as<double>();
        S.lrScale = stu.lrScale.as<float>();
        S.lr = (float)lr;
        ++stu.step;
        S.bc1 = (float)(1.0 - std::pow((double)S.beta1, (double)stu.step));
        S.bc2 = (float)(1.0 - std::pow((double)S.beta2, (double)stu.step));
        launchStudentTrainStep(S, studentGradSmem(stu.maxNin, stu.maxH),
                               stu.maxParams, stream);
        checkLaunch("student training step");
        haveNN = haveNNDeriv = haveE = haveF = false;
        if (lossOut)
        {
            double l[2];
            ck(cudaMemcpyAsync(l, stu.loss.p, sizeof(l), cudaMemcpyDeviceToHost,
                               stream), "read loss");
            ck(cudaStreamSynchronize(stream), "synchronize");
            lossOut[0] = wE * l[0] / batchSize;
            lossOut[1] = wF * l[1] / (3.0 * batchSize);
        }
    }

    void studentRange(bool reset)
    {
        requireStudent(false);
        activate();
        if (reset)
        {
            std::fill(stu.range.begin(), stu.range.end(),
                      Range{DBL_MAX, -DBL_MAX});
            ck(cudaMemcpy(stu.dRange.p, stu.range.data(),
                          sizeof(Range) * stu.range.size(),
                          cudaMemcpyHostToDevice), "reset range");
            stu.haveRange = false;
            return;
        }
        if (!haveSF)
            throw StateError("ERROR: Calculate the symmetry functions "
                             "first.\n");
        RangeLaunch R;
        int const ne = pot.numElements();
        R.maxSF = maxSF;
        R.numElements = ne;
        R.precision = precision;
        for (int e = 0; e < ne; ++e) R.numSF[e] = sfp.numSF[e];
        R.atomsByElem = atomsByElem.as<int>();
        R.es = es;
        R.blkBeg[0] = 0;
        for (int e = 0; e < ne; ++e)
            R.blkBeg[e + 1] = R.blkBeg[e]
                            + (es.start[e + 1] - es.start[e] + 255) / 256;
        for (int e = ne + 1; e <= kMaxElem; ++e) R.blkBeg[e] = R.blkBeg[ne];
        R.G = G.p;
        R.scale = sfScale.as<SFScale>();
        R.range = stu.dRange.as<Range>();
        launchStudentRange(R, stream);
        checkLaunch("training range");
        stu.haveRange = true;
    }

    // Writes the student's weights (n2p2 weights.%03zu.data, the order of
    // NeuralNetwork::setConnections) and its training range.
    void writeStudent(std::string d)
    {
        requireStudent(false);
        if (!d.empty() && d.back() != '/') d += "/";
        activate();
        ck(cudaStreamSynchronize(stream), "synchronize");
        std::vector<float> b(stu.blob.size());
        ck(cudaMemcpy(b.data(), stu.w.p, sizeof(float) * b.size(),
                      cudaMemcpyDeviceToHost), "read student weights");
        ck(cudaMemcpy(stu.range.data(), stu.dRange.p,
                      sizeof(Range) * stu.range.size(),
                      cudaMemcpyDeviceToHost), "read range");
        NNParams const& q = stu.nnp;
        for (int e = 0; e < pot.numElements(); ++e)
        {
            char name[64];
            std::snprintf(name, sizeof(name), "weights.%03d.data",
                          stu.pot.elements[e].atomicNumber);
            std::FILE* f = std::fopen((d + name).c_str(), "w");
            if (!f)
                throw std::runtime_error("ERROR: Cannot write " + d + name
                                         + ".\n");
            std::fprintf(f, "# student weights of element %s (order of "
                            "NeuralNetwork::setConnections)\n",
                         stu.pot.elements[e].symbol.c_str());
            for (int l = 1; l < q.numLayers[e]; ++l)
            {
                int const ni = q.width[e][l - 1], no = q.width[e][l];
                for (int j = 0; j < ni; ++j)
                    for (int k = 0; k < no; ++k)
                        std::fprintf(f, "%24.16E\n",
                                     (double)b[q.woff[e][l] + (long)k * ni + j]);
                for (int k = 0; k < no; ++k)
                    std::fprintf(f, "%24.16E\n", (double)b[q.boff[e][l] + k]);
            }
            std::fclose(f);
        }
        std::FILE* f = std::fopen((d + "training_range.data").c_str(), "w");
        if (!f)
            throw std::runtime_error("ERROR: Cannot write "
                                     + d + "training_range.data.\n");
        std::fprintf(f, "# element SF min max of the unscaled symmetry "
                        "functions over the student's training data\n");
        for (int e = 0; e < pot.numElements(); ++e)
            for (int k = 0; k < sfp.numSF[e]; ++k)
            {
                Range const& r = stu.range[(std::size_t)e * maxSF + k];
                std::fprintf(f, "%d %d %24.16E %24.16E\n", e + 1, k + 1, r.lo,
                             r.hi);
            }
        std::fclose(f);
    }

    void enqueueNN(bool deriv)
    {
        if (stu.mode != 0)
        {
            enqueueGatedStudent(deriv);
            return;
        }
        if (precision != PREC_FP64)
        {
            int const k = (precision == PREC_MIXED) ? 1 : 0;
            if (!tcOk[k])
                throw std::runtime_error("ERROR: The mixed-precision form "
                                         "cannot run this potential: "
                                         + tcWhy[k] + ".\n");
            if (tcGrid[k] == 0)
            {
                ck(cudaDeviceGetAttribute(&smCount,
                                          cudaDevAttrMultiProcessorCount,
                                          device), "device attribute");
                tcGrid[k] = smCount * tcBlocksPerSM(tcp[k]);
            }
            TcNNLaunch T;
            T.n = (int)n;
            T.derivatives = deriv ? 1 : 0;
            T.maxSF = maxSF;
            T.atomsByElem = atomsByElem.as<int>();
            T.es = es;
            T.grid = tcGrid[k];
            T.wblob = tcW[k].as<unsigned char>();
            T.fblob = tcF[k].as<float>();
            T.G = G.as<float>();
            T.energy = Ei.as<double>();
            T.dEdG = dEdG.as<float>();
            T.status = status.as<int>();
            launchNeuralNetworksTC(tcp[k], T, stream);
            return;
        }
        NNLaunch L;
        L.n = (int)n;
        L.derivatives = deriv ? 1 : 0;
        L.maxSF = maxSF;
        L.elem = elem.as<int>();
        L.weights = nnW.as<double>();
        L.G = G.as<double>();
        L.energy = Ei.as<double>();
        L.dEdG = dEdG.as<double>();
        L.status = status.as<int>();
        launchNeuralNetworks(nnp, L, stream);
    }

    void enqueueEnergy()
    {
        if (numStructs > 0)
        {
            BatchEnergyLaunch B;
            B.numStructs = (int)numStructs;
            B.numElements = pot.numElements();
            B.bs = bsDev.as<BatchStruct>();
            B.atomicEnergy = Ei.as<double>();
            B.out = structEnergy.as<double>();
            B.convEnergy = pot.convEnergy;
            B.meanEnergy = pot.meanEnergy;
            B.normalize = pot.normalize ? 1 : 0;
            for (int e = 0; e < pot.numElements(); ++e)
                B.offset[e] = pot.elements[e].atomicEnergyOffset;
            B.status = status.as<int>();
            launchEnergyBatch(B, stream);
            return;
        }
        EnergyLaunch L;
        L.n = (int)n;
        L.atomicEnergy = Ei.as<double>();
        L.out = energyOut.as<double>();
        L.convEnergy = pot.convEnergy;
        L.meanEnergy = pot.meanEnergy;
        L.normalize = pot.normalize ? 1 : 0;
        int const ne = pot.numElements();
        L.numElements = ne;
        for (int e = 0; e < ne; ++e)
        {
            long cnt = es.start[e + 1] - es.start[e];
            L.offsetTerm[e] = cnt * pot.elements[e].atomicEnergyOffset;
        }
        L.status = status.as<int>();
        launchEnergy(L, stream);
    }

    // dG/dr (self) of every atom into dGdrSelf, formed from the stored
    // neighbor slots (the evaluation path never needs it on its own).
    void formSelfDerivatives()
    {
        dGdrSelf.ensure(realBytes() * n * maxSF * 3);
        ForceLaunch L = forceLaunch();
        launchSelfDerivatives(L, dGdrSelf.p, stream);
        checkLaunch("self derivatives");
        ck(cudaStreamSynchronize(stream), "synchronize");
    }

    void enqueueForces()
    {
        ForceLaunch L = forceLaunch();
        L.gather = externalNL ? 0 : 1;
        launchForces(L, stream);
        if (!externalNL) return;
        TargetForceLaunch T;
        T.numLocal = (int)n;
        T.numTargets = (int)numTargets;
        T.revOff = revOff.as<int>();
        T.revEntry = revEntry.as<int>();
        T.selfF = selfF.as<double>();
        T.pairF = pairF.as<double>();
        T.F = Ftarget.as<double>();
        T.forceScale = L.forceScale;
        T.status = status.as<int>();
        launchTargetForces(T, stream);
    }

    ForceLaunch forceLaunch()
    {
        ForceLaunch L;
        int const ne = pot.numElements();
        L.n = (int)n;
        L.numElements = ne;
        L.maxSF = maxSF;
        L.maxSlots = maxSlots;
        L.elem = elem.as<int>();
        L.nbrOff = nbrOff.as<int>();
        L.nbrIdx = nbrIdx.as<int>();
        L.nbrEl = nbrEl.as<int8_t>();
        L.mirror = mirror.as<int>();
        L.slotSF = slotSF.as<int16_t>();
        for (int e = 0; e < ne; ++e)
        {
            L.numSF[e] = sfp.numSF[e];
            for (int f = 0; f < ne; ++f) L.numSlots[e][f] = sfp.numSlots[e][f];
        }
        L.precision = precision;
        L.dEdG = dEdG.p;
        L.dGdr = dGdr.p;
        L.selfF = selfF.as<double>();
        L.pairF = pairF.as<double>();
        L.F = F.as<double>();
        L.forceScale = pot.normalize ? pot.convEnergy / pot.convLength : 1.0;
        L.status = status.as<int>();
        return L;
    }

    // ---- externally supplied neighbor list (InterfaceLammps path) ---------

    // num local atoms (elements), each with counts[i] neighbors: the index
    // of the neighbor in the caller's force array (local atoms first, then
    // ghosts; numTargets in all), its element and r_i - r_neighbor in
    // physical units.  Entries are regrouped by neighbor element (stable),
    // as the symmetry-function kernel stages them.
    void setNeighborList(long num, int32_t const* elems,
                         int64_t const* counts, int64_t const* index,
                         int32_t const* nelems, double const* drIn,
                         long targets)
    {
        requireReady();
        if (num <= 0 || !elems || !counts || targets < num)
            throw std::invalid_argument("ERROR: Invalid neighbor list "
                                        "arguments.\n");
        int const ne = pot.numElements();
        long E = 0;
        for (long i = 0; i < num; ++i)
        {
            if (elems[i] < 0 || elems[i] >= ne || counts[i] < 0)
                throw std::invalid_argument("ERROR: Bad atom in neighbor "
                                            "list.\n");
            E += counts[i];
        }
        if (E > 0 && (!index || !nelems || !drIn))
            throw std::invalid_argument("ERROR: Missing neighbor arrays.\n");
        if (E > 0x7ffffffeL || targets > 0x7ffffffeL)
            throw std::invalid_argument("ERROR: Neighbor list too large.\n");
        activate();
        n = num;
        numStructs = 0;
        externalNL = true;
        numTargets = targets;
        graphValid = false;
        elemHost.assign(elems, elems + num);
        std::vector<int> byElem;
        byElem.reserve(n);
        std::memset(&es, 0, sizeof(es));
        for (int e = 0; e < ne; ++e)
        {
            es.start[e] = (int)byElem.size();
            for (long i = 0; i < n; ++i)
                if (elemHost[i] == e) byElem.push_back((int)i);
        }
        es.start[ne] = (int)byElem.size();
        for (int e = ne + 1; e <= kMaxElem; ++e) es.start[e] = es.start[ne];
        double const L = pot.normalize ? pot.convLength : 1.0;
        std::vector<int> off(n + 1, 0), cntE((std::size_t)n * ne, 0);
        std::vector<int> idx(E), rev((std::size_t)targets + 1, 0);
        std::vector<int8_t> el(E);
        std::vector<double> x(E), y(E), z(E), d(E);
        int maxCnt = 0;
        long src = 0;
        for (long i = 0; i < n; ++i)
        {
            off[i + 1] = off[i] + (int)counts[i];
            maxCnt = std::max(maxCnt, (int)counts[i]);
            long dst = off[i];
            for (int e = 0; e < ne; ++e)
                for (long k = src; k < src + counts[i]; ++k)
                {
                    if (nelems[k] < 0 || nelems[k] >= ne || index[k] < 0
                        || index[k] >= targets)
                        throw std::invalid_argument("ERROR: Bad neighbor "
                                                    "entry.\n");
                    if (nelems[k] != e) continue;
                    double const a = drIn[3 * k], b = drIn[3 * k + 1],
                                 c = drIn[3 * k + 2];
                    idx[dst] = (int)index[k];
                    el[dst] = (int8_t)e;
                    // InterfaceLammps::addNeighbor: n.d = sqrt(d2), scaled
                    // like the components.
                    d[dst] = std::sqrt(a * a + b * b + c * c) * L;
                    x[dst] = a * L;
                    y[dst] = b * L;
                    z[dst] = c * L;
                    ++cntE[(std::size_t)i * ne + e];
                    ++rev[idx[dst] + 1];
                    ++dst;
                }
            src += counts[i];
        }
        for (long m = 0; m < targets; ++m) rev[m + 1] += rev[m];
        std::vector<int> fill(rev.begin(), rev.end() - 1), revE(E);
        for (long e = 0; e < E; ++e) revE[fill[idx[e]]++] = (int)e;
        ensureStructureBuffers();
        capacity = std::max(capacity, std::max(E, 1L));
        ensureEntryBuffers();
        elem.ensure(sizeof(int) * n);
        atomsByElem.ensure(sizeof(int) * n);
        revOff.ensure(sizeof(int) * (targets + 1));
        revEntry.ensure(sizeof(int) * std::max(E, 1L));
        Ftarget.ensure(sizeof(double) * 3 * targets);
        auto up = [&](DevBuf& b, void const* h, std::size_t bytes) {
            if (bytes)
                ck(cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice,
                                   stream), "upload neighbor list");
        };
        up(elem, elemHost.data(), sizeof(int) * n);
        up(atomsByElem, byElem.data(), sizeof(int) * n);
        up(nbrOff, off.data(), sizeof(int) * (n + 1));
        up(nbrCountElem, cntE.data(), sizeof(int) * cntE.size());
        up(nbrIdx, idx.data(), sizeof(int) * E);
        up(nbrEl, el.data(), E);
        up(dx, x.data(), sizeof(double) * E);
        up(dy, y.data(), sizeof(double) * E);
        up(dz, z.data(), sizeof(double) * E);
        up(dd, d.data(), sizeof(double) * E);
        up(revOff, rev.data(), sizeof(int) * (targets + 1));
        up(revEntry, revE.data(), sizeof(int) * E);
        ck(cudaStreamSynchronize(stream), "neighbor list upload");
        invalidate();
        haveNL = true;
        lastMaxNbr = maxCnt;
        sfCap = 0;
        fitSFCap(maxCnt);
        applyTuned();
    }

    void checkLaunch(char const* what)
    {
        ck(cudaGetLastError(), what);
    }

    // Reads the status words (synchronizes the stream).
    int readStatus()
    {
        ck(cudaMemcpyAsync(statusHost, status.p, sizeof(int) * ST_NUM,
                           cudaMemcpyDeviceToHost, stream), "read status");
        ck(cudaStreamSynchronize(stream), "synchronize");
        return statusHost[ST_FLAGS];
    }

    // Runs `stages` (bit 0 NL, 1 SF, 2 NN, 3 E, 4 F) with capacity retries.
    // Staging capacity of the SF kernel: the largest neighbor count plus
    // headroom for the next frames, in multiples of 32.
    void fitSFCap(int maxNbr)
    {
        maxNbr = std::max(maxNbr, lastMaxNbr);
        int const cap = ((std::max(maxNbr, 1) + 8 + 15) / 16) * 16;
        if (sfSharedBytes(sfp, cap, precision) > 227 * 1024)
            throw CapacityError("ERROR: An atom has more neighbors than the "
                                "symmetry-function kernel can stage.\n");
        if (cap > sfCap) graphValid = false;
        sfCap = std::max(cap, sfCap);
    }

    void run(int stages, bool sfDeriv, bool nnDeriv)
    {
        requireReady();
        requireStructure();
        activate();
        ensureStructureBuffers();
        ensureEntryBuffers();
        for (int attempt = 0; attempt < 8; ++attempt)
        {
            enqueueReset();
            int st = stages;
            // Unknown neighbor counts (new structure): run the neighbor list
            // alone first and size the SF staging from its maximum.
            bool const sizing = (st & 1) && (st & 2) && sfCap <= 0;
            if (sizing) st = 1;
            beginProfile();
            if (st & 1) { enqueueNL(); mark(1); }
            if (st & 2)
            {
                enqueueSF(sfDeriv);
                if (ewCheck) enqueueEW();
                mark(2);
            }
            if (st & 4) { enqueueNN(nnDeriv); mark(3); }
            if (st & 8) { enqueueEnergy(); mark(4); }
            if (st & 16) { enqueueForces(); mark(5); }
            endProfile();
            checkLaunch("kernel launch");
            int const flags = readStatus();
            if (st & 1) lastMaxNbr = statusHost[ST_MAX_NBR];
            if (flags & FLAG_NBR_OVERFLOW)
            {
                grow(statusHost[ST_TOTAL_NBR]);
                stages |= 1;
                continue;
            }
            if (flags & FLAG_MIRROR_MISSING)
                throw std::runtime_error("ERROR: Internal: neighbor list is "
                                         "not symmetric.\n");
            if (flags & FLAG_TC_TIMEOUT)
                throw CudaError("ERROR: A tensor-core wait of the NN kernel "
                                "gave up; results are invalid.\n");
            if (flags & FLAG_SF_PATH)
                throw std::runtime_error("ERROR: Internal: symmetry-function "
                                         "kernel without a needed path.\n");
            if (sizing || (flags & FLAG_SF_CAPACITY))
            {
                fitSFCap(statusHost[ST_MAX_NBR]);
                if (sizing)
                {
                    haveNL = true;
                    stages &= ~1;   // the neighbor list of this run stands
                }
                continue;
            }
            if (stages & 1)
            {
                haveNL = true;
                if (sfCap <= 0) fitSFCap(lastMaxNbr);
            }
            if (stages & 2) { haveSF = true; haveSFDeriv = sfDeriv; }
            if (stages & 4) { haveNN = true; haveNNDeriv = nnDeriv; }
            if (stages & 8) haveE = true;
            if (stages & 16) haveF = true;
            if ((stages & 2) && ewCheck) accountEW();
            return;
        }
        throw CapacityError("ERROR: Capacity retries exhausted.\n");
    }

    // Full evaluation enqueued without synchronization (capacities known).
    void enqueueAll(bool forces)
    {
        requireReady();
        requireStructure();
        if (capacity <= 0)
            throw StateError("ERROR: evaluate_async needs known capacities: "
                             "run n2p2b_evaluate once first.\n");
        enqueueReset();
        beginProfile();
        enqueueNL();
        mark(1);
        enqueueSF(forces);
        if (ewCheck) enqueueEW();
        mark(2);
        enqueueNN(forces);
        mark(3);
        enqueueEnergy();
        mark(4);
        if (forces)
        {
            enqueueForces();
            mark(5);
        }
        endProfile();
        checkLaunch("kernel launch");
    }

    int finishStatus()
    {
        int const flags = readStatus();
        if (flags & (FLAG_NBR_OVERFLOW | FLAG_SF_CAPACITY))
            throw CapacityError("ERROR: Capacity exceeded during an "
                                "asynchronous evaluation; call "
                                "n2p2b_evaluate to grow the buffers.\n");
        if (flags & FLAG_MIRROR_MISSING)
            throw std::runtime_error("ERROR: Internal: neighbor list is not "
                                     "symmetric.\n");
        if (flags & FLAG_TC_TIMEOUT)
            throw CudaError("ERROR: A tensor-core wait of the NN kernel gave "
                            "up; results are invalid.\n");
        if (flags & FLAG_SF_PATH)
            throw std::runtime_error("ERROR: Internal: symmetry-function "
                                     "kernel without a needed path.\n");
        haveNL = haveSF = haveNN = haveE = true;
        if (ewCheck) accountEW();
        return 0;
    }

    // ---- CUDA graph of a whole evaluation ----------------------------------

    void captureGraph(bool forces)
    {
        requireReady();
        requireStructure();
        if (capacity <= 0 || sfCap <= 0)
            run(31, forces, forces);       // size every buffer first
        bool const prof = profiling;
        profiling = false;
        // One plain pass fixes the launch configurations (grids, kernel
        // attributes) and proves the capacities fit.
        enqueueAll(forces);
        finishStatus();
        if (graphExec)
        {
            cudaGraphExecDestroy(graphExec);
            graphExec = nullptr;
        }
        graphValid = false;
        cudaGraph_t g = nullptr;
        ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed),
           "begin capture");
        try
        {
            enqueueAll(forces);
        }
        catch (...)
        {
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            profiling = prof;
            throw;
        }
        ck(cudaStreamEndCapture(stream, &g), "end capture");
        cudaError_t const e = cudaGraphInstantiate(&graphExec, g, 0);
        cudaGraphDestroy(g);
        profiling = prof;
        ck(e, "instantiate graph");
        graphValid = true;
        graphForces = forces;
    }

    void launchGraph()
    {
        if (!graphValid || !graphExec)
            throw StateError("ERROR: No valid captured evaluation (capture "
                             "again after changing the structure, buffers "
                             "or settings).\n");
        ck(cudaGraphLaunch(graphExec, stream), "launch graph");
        invalidate();
        haveSFDeriv = haveNNDeriv = haveF = graphForces;
    }

    // ---- autotuner ----------------------------------------------------------

    struct TuneChoice
    {
        int variant, sortCats, nlWarps;
        double ms;
    };
    std::map<std::string, TuneChoice> tuned;

    // Size bucket of the current structure(s): log2 of the atoms per
    // structure, with the precision and the potential's shape.
    std::string tuneKey() const
    {
        long const per = numStructs > 0 ? n / numStructs : n;
        int b = 0;
        while ((2L << b) <= per) ++b;
        return std::to_string(precision) + ":" + std::to_string(maxSF) + ":"
             + std::to_string(b) + (numStructs > 0 ? ":batch" : "");
    }

    void applyTuned()
    {
        auto it = tuned.find(tuneKey());
        if (it == tuned.end())
        {
            // Untuned bucket: the defaults of the next launch.
            sfVariant = -1;
            sfGrid = 0;
            graphValid = false;
            return;
        }
        sfVariant = it->second.variant;
        sfSortCats = it->second.sortCats;
        nlWarpsPerBlock = it->second.nlWarps;
        sfGrid = 0;
        graphValid = false;
    }

    // Times every launch configuration on the current structure(s) and keeps
    // the fastest for this size bucket.
    std::string autotune(bool forces, int reps)
    {
        requireReady();
        requireStructure();
        if (capacity <= 0 || sfCap <= 0) run(31, forces, forces);
        bool const prof = profiling;
        profiling = false;
        std::vector<int> nls = numStructs > 0 ? std::vector<int>{2, 4, 8}
                                              : std::vector<int>{4};
        cudaEvent_t a, b;
        ck(cudaEventCreate(&a), "event");
        ck(cudaEventCreate(&b), "event");
        auto timeIt = [&]() {
            sfGrid = 0;
            enqueueAll(forces);                 // warm
            finishStatus();
            double best = 1e30;
            for (int r = 0; r < reps; ++r)
            {
                ck(cudaEventRecord(a, stream), "record");
                enqueueAll(forces);
                ck(cudaEventRecord(b, stream), "record");
                finishStatus();
                float ms = 0.0f;
                ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
                best = std::min(best, (double)ms);
            }
            return best;
        };
        if (sfVariant < 0)
        {
            sfVariant = sfDefaultVariant(sfp, precision);
            sfSortCats = sfDefaultSort(sfp);
        }
        TuneChoice const start{sfVariant, sfSortCats, nlWarpsPerBlock, 0.0};
        double const t0 = timeIt();
        TuneChoice best{sfVariant, sfSortCats, nlWarpsPerBlock, t0};
        std::string rep;
        for (int v = 0; v < kSFVariants; ++v)
            for (int so : {1, 3, 5, 7})
                for (int w : nls)
                {
                    // The staged kernel ignores the item order.
                    if (v >= 6 && so != 5) continue;
                    sfVariant = v;
                    sfSortCats = so;
                    nlWarpsPerBlock = w;
                    double const t = timeIt();
                    if (t < best.ms) best = TuneChoice{v, so, w, t};
                }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        sfVariant = best.variant;
        sfSortCats = best.sortCats;
        nlWarpsPerBlock = best.nlWarps;
        sfGrid = 0;
        graphValid = false;
        profiling = prof;
        std::string const key = tuneKey();
        tuned[key] = best;
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "bucket %s: sf variant %d, sort %d, nl warps/block %d:"
                      " %.3f ms per evaluation (start %d/%d/%d: %.3f ms)",
                      key.c_str(), best.variant, best.sortCats, best.nlWarps,
                      best.ms, start.variant, start.sortCats, start.nlWarps,
                      t0);
        return buf;
    }

    long totalEntries()
    {
        int off = 0;
        ck(cudaMemcpy(&off, nbrOff.as<int>() + n, sizeof(int),
                      cudaMemcpyDeviceToHost), "read offsets");
        return off;
    }

    // Host permutation from device (element-grouped) order to the
    // reference's list order (j ascending, then image).
    void refOrder(std::vector<int>& off, std::vector<long>& perm)
    {
        if (externalNL)
            throw StateError("ERROR: The neighbor list was supplied by the "
                             "caller.\n");
        long const E = totalEntries();
        off.resize(n + 1);
        ck(cudaMemcpy(off.data(), nbrOff.p, sizeof(int) * (n + 1),
                      cudaMemcpyDeviceToHost), "read offsets");
        std::vector<unsigned long long> k(E);
        if (E > 0)
            ck(cudaMemcpy(k.data(), key.p, sizeof(unsigned long long) * E,
                          cudaMemcpyDeviceToHost), "read keys");
        unsigned long long const mod = (unsigned long long)n
                                     * (numStructs > 0 ? batchNIMG : nlp.nimg);
        perm.resize(E);
        for (long i = 0; i < n; ++i)
        {
            long const b = off[i], e = off[i + 1];
            std::iota(perm.begin() + b, perm.begin() + e, b);
            std::sort(perm.begin() + b, perm.begin() + e,
                      [&](long x, long y) { return k[x] % mod < k[y] % mod; });
        }
    }
};

// ---- C-ABI -----------------------------------------------------------------

namespace
{

template <typename F>
int guarded(n2p2b_context* ctx, F&& f)
{
    if (ctx == nullptr) return N2P2B_ERR_ARGUMENT;
    try
    {
        f();
        ctx->error.clear();
        return N2P2B_OK;
    }
    catch (CudaError const& e)
    {
        ctx->error = e.what();
        return N2P2B_ERR_CUDA;
    }
    catch (CapacityError const& e)
    {
        ctx->error = e.what();
        return N2P2B_ERR_CAPACITY;
    }
    catch (StateError const& e)
    {
        ctx->error = e.what();
        return N2P2B_ERR_STATE;
    }
    catch (ExtrapolationError const& e)
    {
        ctx->error = e.what();
        return N2P2B_ERR_EXTRAPOLATION;
    }
    catch (std::invalid_argument const& e)
    {
        ctx->error = e.what();
        return N2P2B_ERR_ARGUMENT;
    }
    catch (std::exception const& e)
    {
        ctx->error = e.what();
        return N2P2B_ERR_SETUP;
    }
}

} // namespace

extern "C"
{

int n2p2b_create(int device, n2p2b_context** out)
{
    if (out == nullptr) return N2P2B_ERR_ARGUMENT;
    *out = nullptr;
    if (device == -1)
    {
        n2p2b_context* c = new n2p2b_context();
        c->device = -1;
        *out = c;
        return N2P2B_OK;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0
        || device >= count)
        return N2P2B_ERR_CUDA;
    n2p2b_context* c = new n2p2b_context();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess
        || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)
           != cudaSuccess)
    {
        delete c;
        return N2P2B_ERR_CUDA;
    }
    c->ownStream = true;
    *out = c;
    return N2P2B_OK;
}

void n2p2b_destroy(n2p2b_context* ctx)
{
    if (ctx == nullptr) return;
    if (!ctx->hostOnly())
    {
        cudaSetDevice(ctx->device);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    }
    delete ctx;
}

int n2p2b_symmetry_function_params(n2p2b_context const* ctx, int e, int s,
                                   double* out)
{
    if (!ctx || !out || e < 0 || e >= ctx->pot.numElements()) return N2P2B_ERR_ARGUMENT;
    Element const& el = ctx->pot.elements[e];
    if (s < 0 || s >= (int)el.sfs.size()) return N2P2B_ERR_ARGUMENT;
    SymFnc const& f = el.sfs[s];
    double v[10] = {(double)f.type, (double)f.e1, (double)f.e2, f.eta,
                    f.rs, f.rc, f.zeta, f.lambda, f.scalingFactor,
                    (double)f.lineNumber};
    if (isCompactType(f.type))
    {
        // rl, subtype rank (string order: e, p1, p1a, p2, ...), rc,
        // angles in degrees.
        v[3] = f.rl;
        v[4] = f.coreType == CC_EXP ? 0.0
             : (double)(2 * f.coreType - 1 + (f.asymmetric ? 1 : 0));
        v[6] = f.angleLeft;
        v[7] = f.angleRight;
    }
    for (int k = 0; k < 10; ++k) out[k] = v[k];
    return N2P2B_OK;
}

int n2p2b_num_groups(n2p2b_context const* ctx, int e)
{
    if (!ctx || e < 0 || e >= ctx->pot.numElements()) return 0;
    return (int)ctx->pot.elements[e].groups.size();
}

int n2p2b_group_members(n2p2b_context const* ctx, int e, int g, int32_t* idx,
                        int cap)
{
    if (!ctx || e < 0 || e >= ctx->pot.numElements()) return N2P2B_ERR_ARGUMENT;
    auto const& gs = ctx->pot.elements[e].groups;
    if (g < 0 || g >= (int)gs.size()) return N2P2B_ERR_ARGUMENT;
    int const m = (int)gs[g].members.size();
    for (int k = 0; k < m && k < cap; ++k) idx[k] = gs[g].members[k];
    return m;
}

char const* n2p2b_last_error(n2p2b_context const* ctx)
{
    return ctx ? ctx->error.c_str() : "null context";
}

int n2p2b_set_stream(n2p2b_context* ctx, void* stream)
{
    return guarded(ctx, [&] {
        ctx->activate();
        if (ctx->ownStream && ctx->stream)
        {
            cudaStreamSynchronize(ctx->stream);
            cudaStreamDestroy(ctx->stream);
        }
        if (stream)
        {
            ctx->stream = static_cast<cudaStream_t>(stream);
            ctx->ownStream = false;
        }
        else
        {
            ck(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking),
               "cudaStreamCreate");
            ctx->ownStream = true;
        }
    });
}

int n2p2b_set_precision(n2p2b_context* ctx, int mode)
{
    return guarded(ctx, [&] { ctx->setPrecision(mode); });
}

int n2p2b_get_precision(n2p2b_context const* ctx)
{
    return ctx ? ctx->precision : N2P2B_ERR_ARGUMENT;
}

int n2p2b_setup_student(n2p2b_context* ctx, char const* directory)
{
    return guarded(ctx, [&] {
        if (!directory) throw std::invalid_argument("ERROR: directory");
        ctx->setupStudent(directory);
    });
}

int n2p2b_set_student_mode(n2p2b_context* ctx, int mode)
{
    return guarded(ctx, [&] { ctx->setStudentMode(mode); });
}

int n2p2b_get_student_gated_count(n2p2b_context* ctx, int64_t* count)
{
    return guarded(ctx, [&] {
        if (!count) throw std::invalid_argument("ERROR: count");
        ctx->activate();
        *count = ctx->gatedCount();
    });
}

int n2p2b_student_train_step(n2p2b_context* ctx, double const* energy_labels,
                             double const* force_labels, int32_t const* batch,
                             int batch_size, double w_energy, double w_force,
                             double learning_rate, double* loss)
{
    return guarded(ctx, [&] {
        ctx->studentTrainStep(energy_labels, force_labels, batch, batch_size,
                              w_energy, w_force, learning_rate, loss);
    });
}

int n2p2b_student_weights(n2p2b_context* ctx, double* get,
                          double const* set, int64_t* size, int which)
{
    return guarded(ctx, [&] {
        ctx->requireStudent(false);
        ctx->activate();
        std::size_t const m = ctx->stu.blob.size();
        if (size) *size = (int64_t)m;
        DevBuf& b = (which == 1) ? ctx->stu.grad : ctx->stu.w;
        if (which != 0 && which != 1)
            throw std::invalid_argument("ERROR: which");
        std::vector<float> f(m);
        if (get)
        {
            ck(cudaStreamSynchronize(ctx->stream), "synchronize");
            ck(cudaMemcpy(f.data(), b.p, sizeof(float) * m,
                          cudaMemcpyDeviceToHost), "read student weights");
            for (std::size_t k = 0; k < m; ++k) get[k] = f[k];
        }
        if (set)
        {
            if (which != 0)
                throw std::invalid_argument("ERROR: only weights are set");
            for (std::size_t k = 0; k < m; ++k) f[k] = (float)set[k];
            ck(cudaStreamSynchronize(ctx->stream), "synchronize");
            ck(cudaMemcpy(b.p, f.data(), sizeof(float) * m,
                          cudaMemcpyHostToDevice), "write student weights");
            ctx->invalidateNN();
        }
    });
}

int n2p2b_student_reset_optimizer(n2p2b_context* ctx)
{
    return guarded(ctx, [&] {
        ctx->requireStudent(false);
        ctx->activate();
        ctx->resetOptimizer();
    });
}

int n2p2b_student_update_range(n2p2b_context* ctx, int reset)
{
    return guarded(ctx, [&] { ctx->studentRange(reset != 0); });
}

int n2p2b_student_write(n2p2b_context* ctx, char const* directory)
{
    return guarded(ctx, [&] {
        if (!directory) throw std::invalid_argument("ERROR: directory");
        ctx->writeStudent(directory);
    });
}

int n2p2b_setup_symmetry_function_statistics(n2p2b_context* ctx,
                                             int collect_statistics,
                                             int collect_ew, int write_ew,
                                             int stop_on_ew)
{
    return guarded(ctx, [&] {
        if (collect_statistics)
            throw std::invalid_argument("ERROR: Symmetry-function statistics "
                                        "collection is not supported.\n");
        ctx->graphValid = false;
        ctx->ewCheck = collect_ew || write_ew || stop_on_ew;
        ctx->ewWrite = write_ew != 0;
        ctx->ewStop = stop_on_ew != 0;
        ctx->invalidate();
    });
}

int64_t n2p2b_get_num_extrapolation_warnings(n2p2b_context const* ctx)
{
    return ctx ? ctx->ewTotal : 0;
}

int n2p2b_reset_extrapolation_warnings(n2p2b_context* ctx)
{
    return guarded(ctx, [&] { ctx->ewTotal = 0; });
}

int n2p2b_get_extrapolation_counts(n2p2b_context* ctx, int32_t* counts)
{
    return guarded(ctx, [&] {
        if (!ctx->haveEW || !ctx->ewCheck)
            throw StateError("ERROR: No extrapolation check ran (enable it "
                             "with n2p2b_setup_symmetry_function_statistics)."
                             "\n");
        if (counts == nullptr) throw std::invalid_argument("ERROR: counts");
        ctx->activate();
        ck(cudaMemcpy(counts, ctx->ewPerAtom.p, sizeof(int32_t) * ctx->n,
                      cudaMemcpyDeviceToHost), "read warnings");
    });
}

int n2p2b_get_extrapolation_warnings(n2p2b_context* ctx, int64_t capacity,
                                     n2p2b_extrapolation_warning* out,
                                     int64_t* count)
{
    return guarded(ctx, [&] {
        if (!ctx->haveEW || !ctx->ewCheck)
            throw StateError("ERROR: No extrapolation check ran (enable it "
                             "with n2p2b_setup_symmetry_function_statistics)."
                             "\n");
        if (count == nullptr || capacity < 0 || (capacity > 0 && !out))
            throw std::invalid_argument("ERROR: warning buffer");
        ctx->activate();
        std::vector<n2p2b_extrapolation_warning> const w = ctx->ewRecords();
        *count = (int64_t)w.size();
        std::size_t const k = std::min<std::size_t>(w.size(),
                                                    (std::size_t)capacity);
        if (k) std::memcpy(out, w.data(), k * sizeof(w[0]));
    });
}

int n2p2b_load_settings_file(n2p2b_context* ctx, char const* path)
{
    return guarded(ctx, [&] {
        if (path == nullptr) throw std::invalid_argument("ERROR: null path");
        ctx->pot = Potential();
        ctx->generic = ctx->scaled = ctx->weighted = false;
        ctx->tablesReady = false;
        ctx->pot.loadSettingsFile(path);
    });
}

int n2p2b_setup_generic(n2p2b_context* ctx)
{
    return guarded(ctx, [&] {
        ctx->pot.setupGeneric();
        ctx->generic = true;
    });
}

int n2p2b_setup_symmetry_function_scaling(n2p2b_context* ctx,
                                          char const* path)
{
    return guarded(ctx, [&] {
        if (!ctx->generic) throw StateError("ERROR: setupGeneric first.\n");
        if (path) ctx->pot.setupSymmetryFunctionScaling(path);
        else      ctx->pot.setupSymmetryFunctionScalingNone();
        ctx->scaled = true;
        if (ctx->weighted) ctx->buildTables();
    });
}

int n2p2b_setup_neural_network_weights(n2p2b_context* ctx, char const* format)
{
    return guarded(ctx, [&] {
        if (!ctx->generic) throw StateError("ERROR: setupGeneric first.\n");
        if (format == nullptr) throw std::invalid_argument("ERROR: format");
        ctx->pot.setupNeuralNetworkWeights(format);
        ctx->weighted = true;
        if (ctx->scaled) ctx->buildTables();
    });
}

int n2p2b_setup(n2p2b_context* ctx, char const* directory)
{
    if (ctx == nullptr || directory == nullptr) return N2P2B_ERR_ARGUMENT;
    std::string d(directory);
    if (!d.empty() && d.back() != '/') d += "/";
    int rc = n2p2b_load_settings_file(ctx, (d + "input.nn").c_str());
    if (rc) return rc;
    rc = n2p2b_setup_generic(ctx);
    if (rc) return rc;
    rc = n2p2b_setup_symmetry_function_scaling(ctx,
                                               (d + "scaling.data").c_str());
    if (rc) return rc;
    return n2p2b_setup_neural_network_weights(
        ctx, (d + "weights.%03zu.data").c_str());
}

double n2p2b_atomic_energy_offset(n2p2b_context const* ctx, int e)
{
    if (!ctx || e < 0 || e >= ctx->pot.numElements()) return 0.0;
    return ctx->pot.elements[e].atomicEnergyOffset;
}

int n2p2b_atomic_number(n2p2b_context const* ctx, int e)
{
    if (!ctx || e < 0 || e >= ctx->pot.numElements()) return 0;
    return ctx->pot.elements[e].atomicNumber;
}

int n2p2b_unit_conversion(n2p2b_context const* ctx, double* mean_energy,
                          double* conv_energy, double* conv_length)
{
    if (!ctx) return 0;
    bool const nz = ctx->pot.normalize;
    if (mean_energy) *mean_energy = nz ? ctx->pot.meanEnergy : 0.0;
    if (conv_energy) *conv_energy = nz ? ctx->pot.convEnergy : 1.0;
    if (conv_length) *conv_length = nz ? ctx->pot.convLength : 1.0;
    return nz ? 1 : 0;
}

int n2p2b_num_elements(n2p2b_context const* ctx)
{
    return ctx ? ctx->pot.numElements() : 0;
}

int n2p2b_element_symbol(n2p2b_context const* ctx, int e, char* buf,
                         size_t len)
{
    if (!ctx || !buf || e < 0 || e >= ctx->pot.numElements())
        return N2P2B_ERR_ARGUMENT;
    std::snprintf(buf, len, "%s", ctx->pot.elements[e].symbol.c_str());
    return N2P2B_OK;
}

int n2p2b_element_index(n2p2b_context const* ctx, char const* symbol)
{
    if (!ctx || !symbol) return N2P2B_ERR_ARGUMENT;
    for (int e = 0; e < ctx->pot.numElements(); ++e)
        if (ctx->pot.elements[e].symbol == symbol) return e;
    return N2P2B_ERR_ARGUMENT;
}

int n2p2b_num_symmetry_functions(n2p2b_context const* ctx, int e)
{
    if (!ctx || e < 0 || e >= ctx->pot.numElements()) return 0;
    return (int)ctx->pot.elements[e].sfs.size();
}

int n2p2b_num_slots(n2p2b_context const* ctx, int e, int ne)
{
    if (!ctx || e < 0 || ne < 0 || e >= ctx->pot.numElements()
        || ne >= ctx->pot.numElements())
        return 0;
    return (int)ctx->pot.elements[e].sfTable[ne].size();
}

double n2p2b_max_cutoff_radius(n2p2b_context const* ctx)
{
    return ctx ? ctx->pot.maxCutoffRadius : 0.0;
}

int n2p2b_set_structure(n2p2b_context* ctx, int64_t num_atoms,
                        double const* box, double const* positions,
                        int positions_location, int32_t const* elements,
                        int flags)
{
    return guarded(ctx, [&] {
        ctx->setStructure((long)num_atoms, box, positions, positions_location,
                          elements, flags);
    });
}

int n2p2b_set_positions(n2p2b_context* ctx, double const* positions,
                        int positions_location)
{
    return guarded(ctx, [&] {
        if (!positions) throw std::invalid_argument("ERROR: positions");
        ctx->activate();
        ctx->setPositions(positions, positions_location);
    });
}

int n2p2b_calculate_neighbor_list(n2p2b_context* ctx)
{
    return guarded(ctx, [&] { ctx->run(1, false, false); });
}

int n2p2b_calculate_symmetry_function_groups(n2p2b_context* ctx,
                                             int derivatives)
{
    return guarded(ctx, [&] {
        int st = 2;
        if (!ctx->haveNL) st |= 1;
        ctx->run(st, derivatives != 0, false);
    });
}

int n2p2b_calculate_atomic_neural_networks(n2p2b_context* ctx,
                                           int derivatives)
{
    return guarded(ctx, [&] {
        if (!ctx->haveSF)
            throw StateError("ERROR: Symmetry functions not calculated.\n");
        ctx->run(4, ctx->haveSFDeriv, derivatives != 0);
    });
}

int n2p2b_calculate_energy(n2p2b_context* ctx)
{
    return guarded(ctx, [&] {
        if (!ctx->haveNN)
            throw StateError("ERROR: Atomic NNs not calculated.\n");
        ctx->run(8, ctx->haveSFDeriv, ctx->haveNNDeriv);
    });
}

int n2p2b_calculate_forces(n2p2b_context* ctx)
{
    return guarded(ctx, [&] {
        if (!ctx->haveNN || !ctx->haveNNDeriv || !ctx->haveSFDeriv)
            throw StateError("ERROR: Forces need symmetry-function and NN "
                             "derivatives.\n");
        ctx->run(16, true, true);
    });
}

int n2p2b_evaluate(n2p2b_context* ctx, int use_forces)
{
    return guarded(ctx, [&] {
        bool const f = use_forces != 0;
        ctx->run(f ? 31 : 15, f, f);
    });
}

int n2p2b_evaluate_async(n2p2b_context* ctx, int use_forces)
{
    return guarded(ctx, [&] {
        ctx->activate();
        ctx->enqueueAll(use_forces != 0);
        ctx->haveF = use_forces != 0;
        ctx->haveSFDeriv = ctx->haveNNDeriv = use_forces != 0;
    });
}

int n2p2b_finish(n2p2b_context* ctx)
{
    return guarded(ctx, [&] {
        ctx->activate();
        ctx->finishStatus();
    });
}

int n2p2b_get_energy(n2p2b_context* ctx, double* energy)
{
    return guarded(ctx, [&] {
        if (!ctx->haveE) throw StateError("ERROR: Energy not calculated.\n");
        if (!energy) throw std::invalid_argument("ERROR: energy");
        ctx->activate();
        if (ctx->numStructs > 0)
        {
            std::vector<double> e(ctx->numStructs);
            ck(cudaStreamSynchronize(ctx->stream), "synchronize");
            ck(cudaMemcpy(e.data(), ctx->structEnergy.p,
                          sizeof(double) * e.size(), cudaMemcpyDeviceToHost),
               "read energies");
            double t = 0.0;
            for (double v : e) t += v;
            *energy = t;
            return;
        }
        ck(cudaMemcpyAsync(ctx->energyHost, ctx->energyOut.p,
                           sizeof(double) * 2, cudaMemcpyDeviceToHost,
                           ctx->stream), "read energy");
        ck(cudaStreamSynchronize(ctx->stream), "synchronize");
        *energy = ctx->energyHost[1];
    });
}

int n2p2b_set_structures(n2p2b_context* ctx, int64_t num_structures,
                         int64_t const* atom_counts, double const* boxes,
                         double const* positions, int positions_location,
                         int32_t const* elements, int flags)
{
    return guarded(ctx, [&] {
        ctx->setStructures(num_structures, atom_counts, boxes, positions,
                           positions_location, elements, flags);
    });
}

int n2p2b_get_structure_energies(n2p2b_context* ctx, double* energies)
{
    return guarded(ctx, [&] {
        if (!ctx->haveE) throw StateError("ERROR: Energy not calculated.\n");
        if (!energies) throw std::invalid_argument("ERROR: energies");
        ctx->activate();
        ck(cudaStreamSynchronize(ctx->stream), "synchronize");
        if (ctx->numStructs > 0)
        {
            ck(cudaMemcpy(energies, ctx->structEnergy.p,
                          sizeof(double) * ctx->numStructs,
                          cudaMemcpyDeviceToHost), "read energies");
            return;
        }
        ck(cudaMemcpy(ctx->energyHost, ctx->energyOut.p, sizeof(double) * 2,
                      cudaMemcpyDeviceToHost), "read energy");
        energies[0] = ctx->energyHost[1];
    });
}

int n2p2b_capture_graph(n2p2b_context* ctx, int use_forces)
{
    return guarded(ctx, [&] {
        ctx->activate();
        ctx->captureGraph(use_forces != 0);
    });
}

int n2p2b_launch_graph(n2p2b_context* ctx)
{
    return guarded(ctx, [&] {
        ctx->activate();
        ctx->launchGraph();
    });
}

int n2p2b_autotune(n2p2b_context* ctx, int use_forces, int repetitions,
                   char* report, size_t report_len)
{
    return guarded(ctx, [&] {
        ctx->activate();
        std::string const r = ctx->autotune(use_forces != 0,
                                            std::max(1, repetitions));
        if (report && report_len > 0)
        {
            std::strncpy(report, r.c_str(), report_len - 1);
            report[report_len - 1] = '\0';
        }
    });
}

int n2p2b_get_forces(n2p2b_context* ctx, double* forces, int location)
{
    return guarded(ctx, [&] {
        if (!ctx->haveF) throw StateError("ERROR: Forces not calculated.\n");
        if (!forces) throw std::invalid_argument("ERROR: forces");
        if (ctx->externalNL)
            throw StateError("ERROR: With a supplied neighbor list the forces "
                             "are per target: n2p2b_get_target_forces.\n");
        ctx->activate();
        ck(cudaMemcpyAsync(forces, ctx->F.p, sizeof(double) * 3 * ctx->n,
                           location == N2P2B_DEVICE ? cudaMemcpyDeviceToDevice
                                                    : cudaMemcpyDeviceToHost,
                           ctx->stream), "read forces");
        ck(cudaStreamSynchronize(ctx->stream), "synchronize");
    });
}

int n2p2b_set_neighbor_list(n2p2b_context* ctx, int64_t num_atoms,
                            int32_t const* elements,
                            int64_t const* neighbor_counts,
                            int64_t const* neighbor_index,
                            int32_t const* neighbor_elements,
                            double const* dr, int64_t num_targets)
{
    return guarded(ctx, [&] {
        ctx->setNeighborList(num_atoms, elements, neighbor_counts,
                             neighbor_index, neighbor_elements, dr,
                             num_targets);
    });
}

int n2p2b_get_target_forces(n2p2b_context* ctx, double* forces)
{
    return guarded(ctx, [&] {
        if (!ctx->haveF) throw StateError("ERROR: Forces not calculated.\n");
        if (!ctx->externalNL)
            throw StateError("ERROR: No supplied neighbor list.\n");
        if (!forces) throw std::invalid_argument("ERROR: forces");
        ctx->activate();
        ck(cudaStreamSynchronize(ctx->stream), "synchronize");
        ck(cudaMemcpy(forces, ctx->Ftarget.p,
                      sizeof(double) * 3 * ctx->numTargets,
                      cudaMemcpyDeviceToHost), "read forces");
    });
}

int n2p2b_get_atomic_energies(n2p2b_context* ctx, double* energies)
{
    return guarded(ctx, [&] {
        if (!ctx->haveNN) throw StateError("ERROR: NNs not calculated.\n");
        ctx->activate();
        ck(cudaMemcpy(energies, ctx->Ei.p, sizeof(double) * ctx->n,
                      cudaMemcpyDeviceToHost), "read atomic energies");
        if (ctx->pot.normalize)
            for (long i = 0; i < ctx->n; ++i)
                energies[i] /= ctx->pot.convEnergy;
    });
}

int n2p2b_get_neighbor_counts(n2p2b_context* ctx, int64_t* counts)
{
    return guarded(ctx, [&] {
        if (!ctx->haveNL) throw StateError("ERROR: No neighbor list.\n");
        ctx->activate();
        std::vector<int> c(ctx->n);
        ck(cudaMemcpy(c.data(), ctx->nbrCount.p, sizeof(int) * ctx->n,
                      cudaMemcpyDeviceToHost), "read counts");
        for (long i = 0; i < ctx->n; ++i) counts[i] = c[i];
    });
}

int n2p2b_get_neighbor_list(n2p2b_context* ctx, int64_t* index, double* dr,
                            double* d)
{
    return guarded(ctx, [&] {
        if (!ctx->haveNL) throw StateError("ERROR: No neighbor list.\n");
        ctx->activate();
        std::vector<int> off;
        std::vector<long> perm;
        ctx->refOrder(off, perm);
        long const E = (long)perm.size();
        std::vector<int> idx(E);
        std::vector<double> x(E), y(E), z(E), dd(E);
        if (E > 0)
        {
            ck(cudaMemcpy(idx.data(), ctx->nbrIdx.p, sizeof(int) * E,
                          cudaMemcpyDeviceToHost), "read");
            ck(cudaMemcpy(x.data(), ctx->dx.p, sizeof(double) * E,
                          cudaMemcpyDeviceToHost), "read");
            ck(cudaMemcpy(y.data(), ctx->dy.p, sizeof(double) * E,
                          cudaMemcpyDeviceToHost), "read");
            ck(cudaMemcpy(z.data(), ctx->dz.p, sizeof(double) * E,
                          cudaMemcpyDeviceToHost), "read");
            ck(cudaMemcpy(dd.data(), ctx->dd.p, sizeof(double) * E,
                          cudaMemcpyDeviceToHost), "read");
        }
        for (long e = 0; e < E; ++e)
        {
            long const s = perm[e];
            if (index) index[e] = idx[s];
            if (dr)
            {
                dr[3 * e + 0] = x[s];
                dr[3 * e + 1] = y[s];
                dr[3 * e + 2] = z[s];
            }
            if (d) d[e] = dd[s];
        }
    });
}

int n2p2b_get_symmetry_functions(n2p2b_context* ctx, double* G, int stride)
{
    return guarded(ctx, [&] {
        if (!ctx->haveSF) throw StateError("ERROR: No symmetry functions.\n");
        if (stride < ctx->maxSF) throw std::invalid_argument("ERROR: stride");
        ctx->activate();
        std::vector<double> const g =
            ctx->readReal(ctx->G, (std::size_t)ctx->n * ctx->maxSF);
        for (long i = 0; i < ctx->n; ++i)
        {
            int const ns = ctx->sfp.numSF[ctx->elemHost[i]];
            for (int s = 0; s < ns; ++s)
                G[(std::size_t)i * stride + s] = g[(std::size_t)i * ctx->maxSF + s];
        }
    });
}

int n2p2b_get_dEdG(n2p2b_context* ctx, double* out, int stride)
{
    return guarded(ctx, [&] {
        if (!ctx->haveNN || !ctx->haveNNDeriv)
            throw StateError("ERROR: No dE/dG.\n");
        if (stride < ctx->maxSF) throw std::invalid_argument("ERROR: stride");
        ctx->activate();
        std::vector<double> const g =
            ctx->readReal(ctx->dEdG, (std::size_t)ctx->n * ctx->maxSF);
        for (long i = 0; i < ctx->n; ++i)
        {
            int const ns = ctx->sfp.numSF[ctx->elemHost[i]];
            for (int s = 0; s < ns; ++s)
                out[(std::size_t)i * stride + s] =
                    g[(std::size_t)i * ctx->maxSF + s];
        }
    });
}

int n2p2b_get_dGdr(n2p2b_context* ctx, double* self, int sfStride,
                   double* neighbor, int slotStride)
{
    return guarded(ctx, [&] {
        if (!ctx->haveSF || !ctx->haveSFDeriv)
            throw StateError("ERROR: No symmetry-function derivatives.\n");
        if (sfStride < ctx->maxSF || slotStride < ctx->maxSlots)
            throw std::invalid_argument("ERROR: stride");
        ctx->activate();
        long const n = ctx->n;
        int const S = ctx->maxSlots;
        if (self)
        {
            ctx->formSelfDerivatives();
            std::vector<double> const g =
                ctx->readReal(ctx->dGdrSelf, (std::size_t)n * ctx->maxSF * 3);
            for (long i = 0; i < n; ++i)
            {
                int const ns = ctx->sfp.numSF[ctx->elemHost[i]];
                for (int s = 0; s < ns; ++s)
                    for (int c = 0; c < 3; ++c)
                        self[((std::size_t)i * sfStride + s) * 3 + c] =
                            g[((std::size_t)i * ctx->maxSF + s) * 3 + c];
            }
        }
        if (neighbor)
        {
            std::vector<int> off;
            std::vector<long> perm;
            ctx->refOrder(off, perm);
            long const E = (long)perm.size();
            std::vector<double> const g =
                ctx->readReal(ctx->dGdr, (std::size_t)E * S * 3);
            std::vector<int8_t> el(E);
            if (E > 0)
            {
                ck(cudaMemcpy(el.data(), ctx->nbrEl.p, E,
                              cudaMemcpyDeviceToHost), "read elements");
            }
            std::vector<long> atomOf(E);
            for (long i = 0; i < n; ++i)
                for (long e = off[i]; e < off[i + 1]; ++e) atomOf[e] = i;
            for (long e = 0; e < E; ++e)
            {
                long const s = perm[e];
                long const i = atomOf[s];
                long const cnt = off[i + 1] - off[i];
                long const t = s - off[i];
                double const* blk = g.data() + (std::size_t)off[i] * S * 3;
                int const ns = ctx->sfp.numSlots[ctx->elemHost[i]][el[s]];
                for (int k = 0; k < ns; ++k)
                    for (int c = 0; c < 3; ++c)
                        neighbor[((std::size_t)e * slotStride + k) * 3 + c] =
                            blk[((std::size_t)k * 3 + c) * cnt + t];
            }
        }
    });
}

int n2p2b_set_profiling(n2p2b_context* ctx, int enable)
{
    return guarded(ctx, [&] {
        ctx->activate();
        ctx->collectProfile();
        ctx->profiling = enable != 0;
    });
}

int n2p2b_get_stage_times(n2p2b_context* ctx, double* ms, int64_t* runs,
                          int reset)
{
    return guarded(ctx, [&] {
        if (!ms) throw std::invalid_argument("ERROR: ms");
        ctx->activate();
        ctx->collectProfile();
        for (int k = 0; k < 5; ++k) ms[k] = ctx->stageMs[k];
        if (runs) *runs = ctx->stageRuns;
        if (reset)
        {
            for (double& v : ctx->stageMs) v = 0.0;
            ctx->stageRuns = 0;
        }
    });
}

uint64_t n2p2b_kernel_launch_count(void)
{
    return (uint64_t)g_launches.load();
}

int n2p2b_predict(n2p2b_context* ctx, int64_t num_atoms, double const* box,
                  double const* positions, int32_t const* elements,
                  double* energy, double* forces)
{
    int rc = n2p2b_set_structure(ctx, num_atoms, box, positions, N2P2B_HOST,
                                 elements, N2P2B_REMAP);
    if (rc) return rc;
    rc = n2p2b_evaluate(ctx, forces != nullptr);
    if (rc) return rc;
    if (energy)
    {
        rc = n2p2b_get_energy(ctx, energy);
        if (rc) return rc;
    }
    if (forces) rc = n2p2b_get_forces(ctx, forces, N2P2B_HOST);
    return rc;
}

} // extern "C"
