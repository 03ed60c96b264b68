// Updater: host orchestration of one system (the drop-in for UpdaterGPUScBFM_AB_Type).
//
// initialize() follows src/pscbfm/UpdaterGPUScBFM_AB_Type.cu:490-690: bond-set check, colouring,
// per-colour groups in stable original order, neighbour ids re-indexed to sorted slots, lattice
// built from the positions. run() follows CRITICAL.cu:414-698: per MCS nColors sub-steps, each
// drawing (colour, seed) on the host and advancing that colour group on the device.

#include "bfm_engine.hpp"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>

namespace bfm {

void cuda_check(cudaError_t e, char const* what)
{
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CudaError(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    }
}

namespace {

constexpr uint32_t kStepCap = 8192;       // step entries staged per host->device copy
constexpr uint32_t kGraphMcs = 32;        // MCS per captured graph chunk
constexpr uint32_t kSlotAlign = 32;

bool pow2(uint32_t v) { return v && !(v & (v - 1)); }

// UpdaterGPUScBFM_AB_Type.cu:797-848 (the reference's message for a side its bit shifts cannot take)
std::string not_pow2_message(uint32_t bx, uint32_t by, uint32_t bz)
{
    std::ostringstream m;
    m << "[UpdaterGPUScBFM_AB_Type::setLatticeSize] Could not determine value for bit shift. Check whether "
         "the box size is a power of 2 (and at least 4)! ( box="
      << bx << "," << by << "," << bz << " )";
    return m.str();
}

uint32_t ilog2(uint32_t v)
{
    uint32_t l = 0;
    while ((1u << l) < v) ++l;
    return l;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Per-axis contributions of the brick coordinates to the brick index: the bits of the three
// brick coordinates are interleaved x, y, z from the lowest level up (a Z-curve for a cubic box;
// axes that run out of bits drop out of the rotation).
std::vector<uint32_t> brick_tables(uint32_t const nb[3])
{
    std::vector<uint32_t> tab(nb[0] + nb[1] + nb[2]);
    brick_tables_fill(nb, tab.data());
    return tab;
}

inline uint32_t host_brick_pos(uint32_t v, uint32_t a) { return brick_pos(v, a); }

}  // namespace

ArenaLayout arena_layout(uint32_t n, uint32_t npad, uint32_t maxc, uint32_t nwords, uint32_t ntab,
                         uint32_t nColors, uint32_t maxGroup, uint32_t codeMode)
{
    ArenaLayout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t const o = off;
        off = align256(off + bytes);
        return o;
    };
    L.x = take(4ull * npad);
    L.y = take(4ull * npad);
    L.z = take(4ull * npad);
    L.nbr = take(4ull * maxc * npad);
    L.nnb = take(npad);
    L.flags = take(2ull * npad);
    L.mark = take(8ull * npad);
    L.lat = take(8ull * nwords);
    L.tmp = take(16ull * nwords);
    L.tab = take(4ull * ntab);
    L.grp = take(4ull * 2 * nColors);
    L.stats = take(kStatBytes);
    L.desc = take(sizeof(SysDev));
    L.steps = take(sizeof(StepEntry) * (kStepCap + 1));   // the StepGen, then the entries
    L.list = take(4);
    L.gs = take(sizeof(GridSync));
    L.rec = take(codeMode == kCodeNone ? 0 : 4ull * rec_words(codeMode) * npad);
    L.nbrr = take(4ull * maxc * npad);
    L.plane = take(8ull * 768);
    L.moveOk = take(512);
    L.dir = take(4ull * kDirTab);
    // mover lists of the bond-code grid kernels: one segment of kBcTileSpan entries per tile
    L.segs = codeMode == kCodeNone ? 0u : std::max((maxGroup + kBcTileSpan - 1) / kBcTileSpan, 1u);
    L.mlist = take(4ull * 2 * L.segs * kBcTileSpan);
    L.mword = take(4ull * 2 * L.segs * kBcTileSpan);
    L.mcount = take(4ull * 2 * L.segs);
    // position read-back in the caller's order
    L.slotOf = take(4ull * n);
    L.xyzOut = take(12ull * n);
    L.snap = take(8ull * (4 * kSnapRing + 1));   // counter snapshots of graph replays, then their count
    L.bytes = off;
    return L;
}

size_t observables_bytes(uint32_t npad, uint32_t nMol)
{
    return align256(4ull * npad) + align256(8ull * nMol) + align256(12ull * npad) +
           align256(sizeof(long long) * obs_words(nMol));
}

// ============================================================================ construction

Updater::Updater(int gpu)
{
    std::fill(forbidden_, forbidden_ + 512, true);
    setGpu(gpu);
}

Updater::~Updater()
{
    try {
        freeDevice();
    } catch (...) {
    }
    if (stream_) cudaStreamDestroy(stream_);
}

void Updater::setGpu(int gpu)
{
    int count = 0;
    cuda_check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (gpu < 0 || gpu >= count) {
        std::ostringstream m;
        m << "[UpdaterGPUScBFM_AB_Type::setGpu] GPU with ID " << gpu << " not present. Only " << count
          << " GPUs are available.";
        throw std::invalid_argument(m.str());
    }
    if (initialized() && gpu != gpu_) throw std::runtime_error("[setGpu] cannot move an initialized system to another GPU");
    cuda_check(cudaSetDevice(gpu), "cudaSetDevice");
    if (stream_ && gpu != gpu_) {
        cudaStreamDestroy(stream_);
        stream_ = nullptr;
    }
    gpu_ = gpu;
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, gpu), "cudaDeviceGetAttribute");
    smCount_ = (uint32_t)sms;
    if (!stream_) cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
}

void Updater::requireN(char const* who) const
{
    if (!nSet_) throw std::runtime_error(std::string("[") + who + "] setNrOfAllMonomers has not been called");
}

void Updater::requireInit(char const* who) const
{
    if (!initialized()) throw std::runtime_error(std::string("[") + who + "] initialize has not been called");
}

// ============================================================================ setters

void Updater::setPeriodicity(bool px, bool py, bool pz)
{
    // UpdaterGPUScBFM_AB_Type.cu:728-753 accepts fully periodic boxes in its default build and
    // fully non-periodic ones in its NONPERIODICITY build; here every axis chooses on its own.
    if (initialized()) throw std::runtime_error("[setPeriodicity] call it before initialize");
    uint32_t const walls = (px ? 0u : 1u) | (py ? 0u : 2u) | (pz ? 0u : 4u);
    for (int a = 0; a < 3; ++a)
        if (!((walls >> a) & 1u) && box_[a] && !pow2(box_[a]))
            throw std::runtime_error(not_pow2_message(box_[0], box_[1], box_[2]) +
                                     " A periodic axis needs a power-of-two side.");
    walls_ = walls;
}

uint32_t Updater::latticeSide(int a) const
{
    // a periodic axis wraps with the lattice's mask, so its side is the box side (a power of two);
    // a walled axis never wraps (corners stay in [0, L-2]), so its box sits in the lowest cells of
    // a power-of-two lattice side and the walls stay at the box side
    uint32_t const L = box_[a];
    if (!((walls_ >> a) & 1u) || pow2(L)) return L;
    uint32_t P = 4;
    while (P < L) P *= 2;
    return P;
}

void Updater::setNrOfAllMonomers(uint32_t n)
{
    if (n_ != 0 || initialized()) {
        std::ostringstream m;
        m << "[UpdaterGPUScBFM_AB_Type::setNrOfAllMonomers] Number of Monomers already set to " << n_ << "!";
        throw std::runtime_error(m.str());
    }
    n_ = n;
    nSet_ = true;
    xyz_.assign((size_t)n * 3, 0);
    attr_.assign(n, 0);
    nbrCnt_.assign(n, 0);
    nbrIds_.assign((size_t)n * kMaxConn, 0);
}

void Updater::setAttribute(uint32_t i, int32_t a)
{
    requireN("setAttribute");
    if (i >= n_) throw std::out_of_range("[setAttribute] monomer index out of range");
    attr_[i] = a;
}

void Updater::setMonomerCoordinates(uint32_t i, int32_t x, int32_t y, int32_t z)
{
    requireN("setMonomerCoordinates");
    if (i >= n_) throw std::out_of_range("[setMonomerCoordinates] monomer index out of range");
    if (hostStale_) pullPositions();
    xyz_[3 * (size_t)i] = x;
    xyz_[3 * (size_t)i + 1] = y;
    xyz_[3 * (size_t)i + 2] = z;
    if (initialized()) setCoordinates(xyz_.data(), n_);
}

void Updater::setConnectivity(uint32_t a, uint32_t b)
{
    requireN("setConnectivity");
    if (initialized()) throw std::runtime_error("[setConnectivity] bonds are fixed after initialize");
    if (a >= n_ || b >= n_) throw std::out_of_range("[setConnectivity] monomer index out of range");
    // UpdaterGPUScBFM_AB_Type.cu:777-795 (directed: call once per direction)
    if (nbrCnt_[a] >= (uint32_t)kMaxConn) {
        std::ostringstream m;
        m << "[UpdaterGPUScBFM_AB_Type::setConnectivity] The maximum amount of bonds per monomer (" << kMaxConn
          << ") has been exceeded!";
        throw std::invalid_argument(m.str());
    }
    nbrIds_[(size_t)a * kMaxConn + nbrCnt_[a]++] = b;
}

void Updater::setLatticeSize(uint32_t bx, uint32_t by, uint32_t bz)
{
    if (box_[0] == bx && box_[1] == by && box_[2] == bz) return;
    if (initialized()) throw std::runtime_error("[setLatticeSize] the box is fixed after initialize");
    // UpdaterGPUScBFM_AB_Type.cu:797-848; positions are int32 here, boxes up to 1024 per side
    if (bx > 1024 || by > 1024 || bz > 1024) {
        std::ostringstream m;
        m << "[UpdaterGPUScBFM_AB_Type::setLatticeSize] The box size (" << bx << "," << by << "," << bz
          << ") is larger than supported (<= 1024 per side)";
        throw std::invalid_argument(m.str());
    }
    // the reference needs powers of two on every axis; here only periodic axes do (setPeriodicity
    // comes first in the reference's call order, and checks the sides again if it comes later)
    uint32_t const b[3] = {bx, by, bz};
    for (int a = 0; a < 3; ++a)
        if (b[a] < 4 || (!((walls_ >> a) & 1u) && !pow2(b[a])))
            throw std::runtime_error(not_pow2_message(bx, by, bz));
    box_[0] = bx;
    box_[1] = by;
    box_[2] = bz;
}

void Updater::copyBondSet(int dx, int dy, int dz, bool forbidden)
{
    // UpdaterGPUScBFM_AB_Type.cu:693-697 with the index of CRITICAL.cu:243-261
    uint32_t const idx = (uint32_t(dx) & 7u) | ((uint32_t(dy) & 7u) << 3) | ((uint32_t(dz) & 7u) << 6);
    forbidden_[idx] = forbidden;
}

void Updater::populateLattice()
{
    // UpdaterGPUScBFM_AB_Type.cu:850-872 fills the host lattice used by checkSystem; every
    // coordinate maps into the periodic box, so only the preconditions are checked here.
    requireN("populateLattice");
    if (!box_[0]) throw std::runtime_error("[populateLattice] setLatticeSize has not been called");
    latticePopulated_ = true;
}

void Updater::setDrawCounter(uint64_t seed)
{
    drawKind_ = kDrawCounter;
    drawSeed_ = seed;
    drawFn_ = nullptr;
    drawCtx_ = nullptr;
}

void Updater::setSubStep(uint64_t t)
{
    requireInit("setSubStep");
    if (drawKind_ != kDrawCounter) throw std::runtime_error("[setSubStep] only the counter draw stream has a position");
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    scrubPending(stream_);   // pending marks are tied to the parity of the current position
    subStep_ = t;
}

void Updater::setDrawCallback(DrawFn fn, void* ctx)
{
    if (!fn) throw std::invalid_argument("[setDrawCallback] null callback");
    drawKind_ = kDrawCallback;
    drawFn_ = fn;
    drawCtx_ = ctx;
}

void Updater::dropGraphs()
{
    // the captured graphs hold the launches of the old configuration
    if (graphs_.empty()) return;
    if (stream_) cuda_check(cudaStreamSynchronize(stream_), "graph reset");
    for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
    graphs_.clear();
}

void Updater::setGridBlock(int block)
{
    // CTA size of the bond-code check (0: the default)
    if (block != 0 && !check_block_ok(block))
        throw std::invalid_argument("[setGridBlock] the check's CTA size must be 128, 256 or 512 threads");
    if (block == gridBlock_) return;
    dropGraphs();
    gridBlock_ = block;
}

void Updater::setPerformShape(int warps, int group)
{
    if (!perform_shape_ok(warps, group))
        throw std::invalid_argument("[setPerformShape] warps per CTA and per tile must be 1, 2, 4 or 8, the "
                                    "second at most the first (0, 0: the default)");
    if (warps == perfWarps_ && group == perfGroup_) return;
    dropGraphs();
    perfWarps_ = warps;
    perfGroup_ = group;
}

void Updater::setMode(int mode)
{
    if (mode < kModeAuto || mode > kModeCluster) throw std::invalid_argument("[setMode] unknown mode");
    if (mode == kModeResident && initialized() && !residentEligible())
        throw std::invalid_argument("[setMode] this system does not fit the resident kernel");
    mode_ = mode;
}

// ============================================================================ initialize

void Updater::initialize()
{
    if (initialized())
        throw std::runtime_error(
            "[UpdaterGPUScBFM_AB_Type::initialize] Initialize was already called and may not be called again until "
            "cleanup was called!");
    checkSetup();
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");

    // colouring and groups (UpdaterGPUScBFM_AB_Type.cu:549-608)
    colour_ = colour_bond_graph(n_, nbrCnt_.data(), nbrIds_.data(), kMaxConn);
    uint32_t nC = 0;
    for (uint8_t c : colour_) nC = std::max(nC, (uint32_t)c + 1);
    grpSize_.assign(nC, 0);
    for (uint8_t c : colour_) ++grpSize_[c];
    grpOff_.assign(nC, 0);
    uint32_t acc = 0;
    maxGroup_ = 0;
    for (uint32_t c = 0; c < nC; ++c) {
        grpOff_[c] = acc;
        acc += (grpSize_[c] + kSlotAlign - 1) / kSlotAlign * kSlotAlign;
        maxGroup_ = std::max(maxGroup_, grpSize_[c]);
    }
    npad_ = std::max(acc, kSlotAlign);
    oldToNew_.assign(n_, 0);
    {
        std::vector<uint32_t> next = grpOff_;
        for (uint32_t i = 0; i < n_; ++i) oldToNew_[i] = next[colour_[i]]++;
    }
    maxc_ = 1;
    for (uint32_t i = 0; i < n_; ++i) maxc_ = std::max(maxc_, nbrCnt_[i]);

    // host images
    uint32_t const P[3] = {latticeSide(0), latticeSide(1), latticeSide(2)};
    uint32_t nb[3] = {P[0] / 4, P[1] / 4, P[2] / 4};
    uint32_t const nwords = nb[0] * nb[1] * nb[2];
    std::vector<uint32_t> tab = brick_tables(nb);
    std::vector<int32_t> hx(npad_, kPadCoord), hy(npad_, 0), hz(npad_, 0);
    std::vector<uint32_t> hnbr((size_t)maxc_ * npad_, 0);
    std::vector<uint8_t> hnnb(npad_, 0);
    std::vector<unsigned long long> hlat(nwords, 0ull);
    for (uint32_t i = 0; i < n_; ++i) {
        uint32_t const s = oldToNew_[i];
        int32_t const x = xyz_[3 * (size_t)i], y = xyz_[3 * (size_t)i + 1], z = xyz_[3 * (size_t)i + 2];
        hx[s] = x;
        hy[s] = y;
        hz[s] = z;
        hnnb[s] = (uint8_t)nbrCnt_[i];
        for (uint32_t k = 0; k < nbrCnt_[i]; ++k)
            hnbr[(size_t)k * npad_ + s] = oldToNew_[nbrIds_[(size_t)i * kMaxConn + k]];
        uint32_t const mx = uint32_t(x) & (P[0] - 1), my = uint32_t(y) & (P[1] - 1), mz = uint32_t(z) & (P[2] - 1);
        uint32_t const w = tab[mx >> 2] + tab[nb[0] + (my >> 2)] + tab[nb[0] + nb[1] + (mz >> 2)];
        uint32_t const b = host_brick_pos(mx & 3, 0) | host_brick_pos(my & 3, 1) | host_brick_pos(mz & 3, 2);
        hlat[w] |= 1ull << b;
    }
    std::vector<uint32_t> hgrp(2 * (size_t)nC);
    for (uint32_t c = 0; c < nC; ++c) {
        hgrp[2 * c] = grpOff_[c];
        hgrp[2 * c + 1] = grpSize_[c];
    }
    // bond-code representation: symmetric neighbour lists (every i->j has a j->i partner, the
    // m-th occurrence of j in i's list pairing with the m-th occurrence of i in j's) and <= 6
    // bonds per monomer
    codeMode_ = kCodeNone;
    // (mover-list entries hold a slot in 27 bits)
    if (repr_ == kReprAuto && maxc_ <= 6 && npad_ < (1u << 27)) {
        bool sym = true;
        for (uint32_t i = 0; i < n_ && sym; ++i)
            for (uint32_t k = 0; k < nbrCnt_[i] && sym; ++k) {
                uint32_t const j = nbrIds_[(size_t)i * kMaxConn + k];
                uint32_t occ = 0, want = 0, seen = 0;
                for (uint32_t q = 0; q < k; ++q) occ += nbrIds_[(size_t)i * kMaxConn + q] == j ? 1 : 0;
                for (uint32_t q = 0; q < nbrCnt_[j]; ++q) want += nbrIds_[(size_t)j * kMaxConn + q] == i ? 1 : 0;
                for (uint32_t q = 0; q < nbrCnt_[i]; ++q) seen += nbrIds_[(size_t)i * kMaxConn + q] == j ? 1 : 0;
                sym = want == seen && occ < want;
            }
        if (sym) codeMode_ = maxc_ <= 3 ? kCode32 : kCode64;
    }
    std::vector<uint32_t> hpk;
    std::vector<uint8_t> hcode;
    std::vector<uint32_t> hnbrr;
    std::vector<uint32_t> hrec;

    // one arena for every device array of this system
    ArenaLayout const L = arena_layout(n_, npad_, maxc_, nwords, (uint32_t)tab.size(), nC, maxGroup_, codeMode_);
    uint32_t const segs = L.segs;
    Device d;
    d.bytes = L.bytes;
    // stream-ordered: freeing it later does not wait for the whole device
    cuda_check(cudaMallocAsync(&d.arena, L.bytes, stream_), "cudaMallocAsync(system arena)");
    char* base = static_cast<char*>(d.arena);
    dev_ = d;
    SysDev& h = dev_.h;
    h.x = reinterpret_cast<int32_t*>(base + L.x);
    h.y = reinterpret_cast<int32_t*>(base + L.y);
    h.z = reinterpret_cast<int32_t*>(base + L.z);
    h.nbr = reinterpret_cast<uint32_t*>(base + L.nbr);
    h.nnb = reinterpret_cast<uint8_t*>(base + L.nnb);
    h.flags = reinterpret_cast<uint8_t*>(base + L.flags);
    h.tmark = reinterpret_cast<uint32_t*>(base + L.mark);
    h.lat = reinterpret_cast<unsigned long long*>(base + L.lat);
    h.tmp = reinterpret_cast<unsigned long long*>(base + L.tmp);
    h.brickTab = reinterpret_cast<uint32_t*>(base + L.tab);
    h.grp = reinterpret_cast<uint32_t*>(base + L.grp);
    h.stats = reinterpret_cast<unsigned long long*>(base + L.stats);
    h.npad = npad_;
    h.nwords = nwords;
    h.maxc = maxc_;
    h.nColors = nC;
    for (int a = 0; a < 3; ++a) {
        h.mask[a] = P[a] - 1;
        h.lim[a] = box_[a] - 1;
        h.nb[a] = nb[a];
    }
    brick_params(nb, h.mb, h.hx, h.hy);
    for (uint32_t a = 0; a < 3; ++a) h.amask[a] = axis_address_mask(a, nb, tab.data());
    std::memset(h.forbid, 0, sizeof(h.forbid));
    for (uint32_t i = 0; i < 512; ++i)
        if (forbidden_[i]) h.forbid[i >> 5] |= 1u << (i & 31);
    dev_.dDesc = reinterpret_cast<SysDev*>(base + L.desc);
    h.gen = reinterpret_cast<StepGen*>(base + L.steps);
    dev_.dSteps = reinterpret_cast<StepEntry*>(base + L.steps) + 1;
    dev_.stepCap = kStepCap;
    dev_.dList = reinterpret_cast<uint32_t*>(base + L.list);
    dev_.gs = reinterpret_cast<GridSync*>(base + L.gs);
    dev_.slotOf = reinterpret_cast<uint32_t*>(base + L.slotOf);
    dev_.xyzOut = reinterpret_cast<int32_t*>(base + L.xyzOut);
    dev_.snap = reinterpret_cast<unsigned long long*>(base + L.snap);
    dev_.snapSeq = dev_.snap + 4 * kSnapRing;
    h.rec = codeMode_ == kCodeNone ? nullptr : reinterpret_cast<uint32_t*>(base + L.rec);
    h.nbrr = reinterpret_cast<uint32_t*>(base + L.nbrr);
    h.planeTab = reinterpret_cast<unsigned long long*>(base + L.plane);
    h.moveOk = reinterpret_cast<uint8_t*>(base + L.moveOk);
    h.dirTab = reinterpret_cast<uint32_t*>(base + L.dir);
    h.mlist = reinterpret_cast<uint32_t*>(base + L.mlist);
    h.mword = reinterpret_cast<uint32_t*>(base + L.mword);
    h.mcount = reinterpret_cast<uint32_t*>(base + L.mcount);
    h.listStride = segs * kBcTileSpan;
    h.countStride = segs;
    h.codeMode = codeMode_;
    h.walls = walls_;

    cudaStream_t s = stream_;
    std::vector<unsigned long long> hplane(768);
    plane_table_fill(hplane.data());
    std::vector<uint8_t> hmove(512);
    move_ok_fill(forbidden_, hmove.data());
    // index 0 (the zero vector) is never a bond of a valid state: its entry allows every direction,
    // so the unused (zero) fields of a code word drop out of the AND over all fields
    hmove[0] = 0x3F;
    std::vector<uint32_t> hdir(kDirTab);
    uint32_t const hi[3] = {box_[0] - 2, box_[1] - 2, box_[2] - 2};   // walls at the box sides
    dir_table_fill(nb, tab.data(), hi, walls_, hdir.data());
    cuda_check(cudaMemcpyAsync(const_cast<unsigned long long*>(h.planeTab), hplane.data(), 8ull * 768,
                               cudaMemcpyHostToDevice, s), "upload plane table");
    cuda_check(cudaMemcpyAsync(const_cast<uint8_t*>(h.moveOk), hmove.data(), 512, cudaMemcpyHostToDevice, s),
               "upload move table");
    cuda_check(cudaMemcpyAsync(const_cast<uint32_t*>(h.dirTab), hdir.data(), 4ull * hdir.size(),
                               cudaMemcpyHostToDevice, s), "upload direction table");
    if (codeMode_ != kCodeNone) {
        hostCodes(hpk, hcode, hnbrr);
        hrec = slotRecords(hpk, hcode);
        cuda_check(cudaMemcpyAsync(h.rec, hrec.data(), 4ull * hrec.size(), cudaMemcpyHostToDevice, s),
                   "upload slot records");
        cuda_check(cudaMemcpyAsync(const_cast<uint32_t*>(h.nbrr), hnbrr.data(), 4ull * hnbrr.size(),
                                   cudaMemcpyHostToDevice, s), "upload nbrr");
    }
    if (codeMode_ != kCodeNone) toImageOffsets(hx, hy, hz);
    cuda_check(cudaMemcpyAsync(h.x, hx.data(), 4ull * npad_, cudaMemcpyHostToDevice, s), "upload x");
    cuda_check(cudaMemcpyAsync(h.y, hy.data(), 4ull * npad_, cudaMemcpyHostToDevice, s), "upload y");
    cuda_check(cudaMemcpyAsync(h.z, hz.data(), 4ull * npad_, cudaMemcpyHostToDevice, s), "upload z");
    cuda_check(cudaMemcpyAsync(const_cast<uint32_t*>(h.nbr), hnbr.data(), 4ull * maxc_ * npad_,
                               cudaMemcpyHostToDevice, s), "upload nbr");
    cuda_check(cudaMemcpyAsync(const_cast<uint8_t*>(h.nnb), hnnb.data(), npad_, cudaMemcpyHostToDevice, s),
               "upload nnb");
    cuda_check(cudaMemsetAsync(h.flags, 0, 2ull * npad_, s), "memset flags");
    cuda_check(cudaMemsetAsync(h.tmark, 0xFF, 8ull * npad_, s), "memset tmark");
    cuda_check(cudaMemcpyAsync(h.lat, hlat.data(), 8ull * nwords, cudaMemcpyHostToDevice, s), "upload lattice");
    cuda_check(cudaMemsetAsync(h.tmp, 0, 16ull * nwords, s), "memset tmp");
    cuda_check(cudaMemcpyAsync(const_cast<uint32_t*>(h.brickTab), tab.data(), 4ull * tab.size(),
                               cudaMemcpyHostToDevice, s), "upload brick table");
    cuda_check(cudaMemcpyAsync(const_cast<uint32_t*>(h.grp), hgrp.data(), 4ull * hgrp.size(),
                               cudaMemcpyHostToDevice, s), "upload groups");
    if (n_) cuda_check(cudaMemcpyAsync(dev_.slotOf, oldToNew_.data(), 4ull * n_, cudaMemcpyHostToDevice, s),
                       "upload slot order");
    cuda_check(cudaMemsetAsync(h.stats, 0, kStatBytes, s), "memset stats");
    cuda_check(cudaMemcpyAsync(dev_.dDesc, &h, sizeof(SysDev), cudaMemcpyHostToDevice, s), "upload descriptor");
    cuda_check(cudaMemsetAsync(dev_.dList, 0, 4, s), "memset list");
    cuda_check(cudaMemsetAsync(dev_.gs, 0, sizeof(GridSync), s), "memset grid barrier");
    cuda_check(cudaMemsetAsync(h.gen, 0, sizeof(StepGen), s), "memset step producer");   // off
    cuda_check(cudaMemsetAsync(dev_.snap, 0, 8ull * (4 * kSnapRing + 1), s), "memset snapshots");
    if (segs) {
        cuda_check(cudaMemsetAsync(h.mcount, 0, 4ull * 2 * segs, s), "memset mover counts");
        // the grid perform loads list slots past a list's end and ignores them: they start as zeros
        cuda_check(cudaMemsetAsync(h.mlist, 0, 4ull * 2 * segs * kBcTileSpan, s), "memset mover lists");
        cuda_check(cudaMemsetAsync(h.mword, 0, 4ull * 2 * segs * kBcTileSpan, s), "memset mover targets");
    }
    if (!stepsFree_) cuda_check(cudaEventCreateWithFlags(&stepsFree_, cudaEventDisableTiming), "cudaEventCreate");
    if (!batchOnly_) ensureStaging();
    cuda_check(cudaStreamSynchronize(s), "initialize");
    buildObservables();
    planCluster();
    subStep_ = 0;
    mcsDone_ = 0;
    lastColor_ = kNoColor;
    hostStale_ = false;
    chainValid_ = false;
    genOn_ = 0;
    snapIssued_ = 0;
    lastRunSnap_ = false;
    lastRunLead_ = false;
    snapMode_ = false;
    pendingTickets_.clear();
}

void Updater::hostCodes(std::vector<uint32_t>& pk, std::vector<uint8_t>& code, std::vector<uint32_t>& nbrr) const
{
    // lattice addresses, bond-code words and neighbour slots with their reverse slot, all in
    // sorted order, from the host positions
    uint32_t const P[3] = {latticeSide(0), latticeSide(1), latticeSide(2)};
    uint32_t const nb[3] = {P[0] / 4, P[1] / 4, P[2] / 4};
    std::vector<uint32_t> const tab = brick_tables(nb);
    pk.assign(npad_, 0u);
    size_t const w = codeMode_ == kCode64 ? 8 : 4;
    uint32_t const countShift = codeMode_ == kCode64 ? 54 : 27;
    code.assign(w * npad_, 0);
    nbrr.assign((size_t)maxc_ * npad_, 0u);
    for (uint32_t i = 0; i < n_; ++i) {
        uint32_t const s = oldToNew_[i];
        int32_t const* p = &xyz_[3 * (size_t)i];
        pk[s] = lattice_address(uint32_t(p[0]) & (P[0] - 1), uint32_t(p[1]) & (P[1] - 1), uint32_t(p[2]) & (P[2] - 1),
                                nb, tab.data());
        uint64_t c = (uint64_t)nbrCnt_[i] << countShift;
        for (uint32_t k = 0; k < nbrCnt_[i]; ++k) {
            uint32_t const j = nbrIds_[(size_t)i * kMaxConn + k];
            int32_t const* q = &xyz_[3 * (size_t)j];
            uint64_t const f = (uint32_t(q[0] - p[0]) & 7u) | ((uint32_t(q[1] - p[1]) & 7u) << 3) |
                               ((uint32_t(q[2] - p[2]) & 7u) << 6);
            c |= f << (9 * k);
            // reverse slot: the occurrence of i in j's list with the same rank as this j in i's
            uint32_t occ = 0;
            for (uint32_t m = 0; m < k; ++m) occ += nbrIds_[(size_t)i * kMaxConn + m] == j ? 1 : 0;
            uint32_t r = 0;
            for (uint32_t m = 0; m < nbrCnt_[j]; ++m)
                if (nbrIds_[(size_t)j * kMaxConn + m] == i) {
                    if (occ == 0) {
                        r = m;
                        break;
                    }
                    --occ;
                }
            nbrr[(size_t)k * npad_ + s] = oldToNew_[j] | (r << kSlotShift);
        }
        std::memcpy(&code[w * s], &c, w);
    }
}

std::vector<uint32_t> Updater::slotRecords(std::vector<uint32_t> const& pk, std::vector<uint8_t> const& code) const
{
    // the records of every slot (SlotRec; padding: zeros): the lattice address in the first word,
    // the code word in the second half
    uint32_t const rw = rec_words(codeMode_);
    size_t const w = codeMode_ == kCode64 ? 8 : 4;
    std::vector<uint32_t> r((size_t)rw * npad_, 0u);
    for (uint32_t g = 0; g < npad_; ++g) {
        r[(size_t)g * rw] = pk[g];
        std::memcpy(&r[(size_t)g * rw + rw / 2], &code[w * g], w);
    }
    return r;
}

std::vector<uint32_t> Updater::moleculeRoots() const
{
    std::vector<uint32_t> parent(n_);
    for (uint32_t i = 0; i < n_; ++i) parent[i] = i;
    auto find = [&](uint32_t a) {
        while (parent[a] != a) a = parent[a] = parent[parent[a]];
        return a;
    };
    for (uint32_t i = 0; i < n_; ++i)
        for (uint32_t k = 0; k < nbrCnt_[i]; ++k) {
            uint32_t a = find(i), b = find(nbrIds_[(size_t)i * kMaxConn + k]);
            if (a != b) parent[a < b ? b : a] = a < b ? a : b;
        }
    for (uint32_t i = 0; i < n_; ++i) parent[i] = find(i);
    return parent;
}

uint32_t Updater::countMolecules() const
{
    std::vector<uint32_t> const root = moleculeRoots();
    uint32_t m = 0;
    for (uint32_t i = 0; i < n_; ++i) m += root[i] == i ? 1u : 0u;
    return m;
}

void Updater::buildObservables()
{
    // molecules: connected components of the bond graph, numbered in order of their lowest id
    std::vector<uint32_t> const root = moleculeRoots();
    std::vector<uint32_t> molOf(n_), rootMol(n_, kNoColor);
    nMol_ = 0;
    molSize_.clear();
    std::vector<uint32_t> first, last;
    for (uint32_t i = 0; i < n_; ++i) {
        uint32_t const r = root[i];
        if (rootMol[r] == kNoColor) {
            rootMol[r] = nMol_++;
            molSize_.push_back(0);
            first.push_back(i);
            last.push_back(i);
        }
        uint32_t const m = rootMol[r];
        molOf[i] = m;
        ++molSize_[m];
        last[m] = i;
    }
    std::vector<uint32_t> molOfSlot(npad_, kNoColor), ends(2ull * nMol_);
    for (uint32_t i = 0; i < n_; ++i) molOfSlot[oldToNew_[i]] = molOf[i];
    for (uint32_t m = 0; m < nMol_; ++m) {
        ends[2 * m] = oldToNew_[first[m]];
        ends[2 * m + 1] = oldToNew_[last[m]];
    }
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t const o = off;
        off = align256(off + bytes);
        return o;
    };
    size_t const oMol = take(4ull * npad_), oEnds = take(8ull * nMol_), oR = take(12ull * npad_);
    size_t const oOut = take(sizeof(long long) * obs_words(nMol_));
    if (off != observables_bytes(npad_, nMol_)) throw std::logic_error("[buildObservables] arena size mismatch");
    cuda_check(cudaMallocAsync(&obsArena_, off, stream_), "cudaMallocAsync(observables)");
    char* base = static_cast<char*>(obsArena_);
    obs_.molOfSlot = reinterpret_cast<uint32_t*>(base + oMol);
    obs_.ends = reinterpret_cast<uint32_t*>(base + oEnds);
    obs_.rx = reinterpret_cast<int32_t*>(base + oR);
    obs_.ry = obs_.rx + npad_;
    obs_.rz = obs_.ry + npad_;
    obs_.nMol = nMol_;
    dObsOut_ = reinterpret_cast<long long*>(base + oOut);
    cuda_check(cudaMemcpyAsync(const_cast<uint32_t*>(obs_.molOfSlot), molOfSlot.data(), 4ull * npad_,
                               cudaMemcpyHostToDevice, stream_), "upload molecules");
    cuda_check(cudaMemcpyAsync(const_cast<uint32_t*>(obs_.ends), ends.data(), 8ull * nMol_, cudaMemcpyHostToDevice,
                               stream_), "upload molecule ends");
    cuda_check(cudaStreamSynchronize(stream_), "observables set-up");
    resetReference();
}

std::vector<uint32_t> Updater::moleculeSizes() const
{
    requireInit("moleculeSizes");
    return molSize_;
}

void Updater::toImageOffsets(std::vector<int32_t>& hx, std::vector<int32_t>& hy, std::vector<int32_t>& hz) const
{
    // padding slots keep kPadCoord, whose low bits are zero
    uint32_t const P[3] = {latticeSide(0), latticeSide(1), latticeSide(2)};
    for (uint32_t g = 0; g < npad_; ++g) {
        hx[g] = image_offset(hx[g], P[0]);
        hy[g] = image_offset(hy[g], P[1]);
        hz[g] = image_offset(hz[g], P[2]);
    }
}

void Updater::resetReference()
{
    requireInit("resetReference");
    if (codeMode_ != kCodeNone) {
        cuda_check(launch_unfold_positions(dev_.dDesc, npad_, const_cast<int32_t*>(obs_.rx), const_cast<int32_t*>(obs_.ry),
                                           const_cast<int32_t*>(obs_.rz), stream_),
                   "reference positions");
        return;
    }
    cuda_check(cudaMemcpyAsync(const_cast<int32_t*>(obs_.rx), dev_.h.x, 4ull * npad_, cudaMemcpyDeviceToDevice, stream_),
               "reference x");
    cuda_check(cudaMemcpyAsync(const_cast<int32_t*>(obs_.ry), dev_.h.y, 4ull * npad_, cudaMemcpyDeviceToDevice, stream_),
               "reference y");
    cuda_check(cudaMemcpyAsync(const_cast<int32_t*>(obs_.rz), dev_.h.z, 4ull * npad_, cudaMemcpyDeviceToDevice, stream_),
               "reference z");
}

void Updater::enqueueObservables(long long* dOut, cudaStream_t s)
{
    requireInit("observables");
    cuda_check(launch_observables(dev_.dDesc, obs_, dOut, npad_, s), "observables");
    ++launches_;
}

void Updater::observablesAsync(long long* hostPinned)
{
    enqueueObservables(dObsOut_, stream_);
    cuda_check(cudaMemcpyAsync(hostPinned, dObsOut_, sizeof(long long) * obs_words(nMol_), cudaMemcpyDeviceToHost,
                               stream_),
               "download observables");
}

void Updater::observables(long long* out)
{
    enqueueObservables(dObsOut_, stream_);
    cuda_check(cudaMemcpyAsync(out, dObsOut_, sizeof(long long) * obs_words(nMol_), cudaMemcpyDeviceToHost, stream_),
               "download observables");
    cuda_check(cudaStreamSynchronize(stream_), "observables");
}

void Updater::checkSetup() const
{
    requireN("initialize");
    if (n_ == 0) throw std::runtime_error("[initialize] the system has no monomers");
    if (!box_[0]) throw std::runtime_error("[initialize] setLatticeSize has not been called");
    for (int a = 0; a < 3; ++a)
        if (!((walls_ >> a) & 1u) && !pow2(box_[a]))
            throw std::runtime_error(not_pow2_message(box_[0], box_[1], box_[2]));
    uint32_t nAllowed = 0;
    for (bool f : forbidden_) nAllowed += f ? 0 : 1;
    if (nAllowed != 108) {
        std::ostringstream m;
        m << "[UpdaterGPUScBFM_AB_Type::initialize] Wrong bond-set! Expected 108 allowed bonds, but got " << nAllowed;
        throw std::runtime_error(m.str());
    }
    // along an axis with walls every corner must lie in [0, L-2] (the cube inside the box)
    for (uint32_t i = 0; i < n_; ++i)
        for (int a = 0; a < 3; ++a)
            if (((walls_ >> a) & 1u) && uint32_t(xyz_[3ull * i + a]) >= box_[a] - 1u) {
                std::ostringstream m;
                m << "[initialize] monomer " << i << " lies outside the walls of the box along axis " << a;
                throw std::runtime_error(m.str());
            }
}

void Updater::copySetup(Updater const& o)
{
    if (initialized()) throw std::runtime_error("[copySetup] target already initialized");
    n_ = o.n_;
    nSet_ = o.nSet_;
    if (o.hostStale_) throw std::runtime_error("[copySetup] source positions are on the device");
    xyz_ = o.xyz_;
    attr_ = o.attr_;
    nbrCnt_ = o.nbrCnt_;
    nbrIds_ = o.nbrIds_;
    for (int a = 0; a < 3; ++a) box_[a] = o.box_[a];
    walls_ = o.walls_;
    std::copy(o.forbidden_, o.forbidden_ + 512, forbidden_);
    latticePopulated_ = o.latticePopulated_;
    drawKind_ = o.drawKind_;
    drawSeed_ = o.drawSeed_;
    drawFn_ = o.drawFn_;
    drawCtx_ = o.drawCtx_;
    mode_ = o.mode_;
    repr_ = o.repr_;
}

uint32_t Updater::maxNeighbours() const
{
    uint32_t m = 0;
    for (uint32_t c : nbrCnt_) m = std::max(m, c);
    return m;
}

void Updater::setRepresentation(int r)
{
    if (r != kReprAuto && r != kReprGather) throw std::invalid_argument("[setRepresentation] unknown representation");
    if (initialized()) throw std::runtime_error("[setRepresentation] must be chosen before initialize");
    repr_ = r;
}

uint32_t Updater::gridTiles() const
{
    uint32_t const span = codeMode_ == kCodeNone ? kGridBlock : kBcTileSpan;
    return std::max((maxGroup_ + span - 1) / span, 1u);
}

cudaError_t Updater::launchCheck(StepEntry const* e, cudaStream_t s, unsigned long long* snap) const
{
    if (codeMode_ == kCodeNone) return launch_check(dev_.dDesc, nullptr, gridTiles(), kGridBlock, e, s);
    return launch_check_bc(dev_.h, dev_.dDesc, nullptr, gridTiles(), e, codeMode_, s, -1, gridBlock_, snap);
}

cudaError_t Updater::launchPerform(StepEntry const* e, cudaStream_t s, PerformArgs pa) const
{
    if (codeMode_ == kCodeNone) return launch_perform(dev_.dDesc, nullptr, gridTiles(), kGridBlock, e, s, pa.next);
    pa.warps = perfWarps_;
    pa.group = perfGroup_;
    return launch_perform_bc(dev_.h, dev_.dDesc, nullptr, gridTiles(), e, codeMode_, s, -1, pa);
}

PerformArgs Updater::performArgs(StepEntry const& e)
{
    // what the host knows of the sub-step: its parity, and whether the previous sub-step left marks
    PerformArgs pa;
    pa.parity = e.parity;
    pa.scope = (e.color != kNoColor ? kPerfCur : 0u) | (e.prevColor != kNoColor ? kPerfPrev : 0u);
    return pa;
}

size_t Updater::residentSmem() const
{
    uint32_t const ntab = dev_.h.nb[0] + dev_.h.nb[1] + dev_.h.nb[2];
    return codeMode_ == kCodeNone ? resident_smem_bytes(dev_.h.nwords, ntab)
                                  : resident_bc_smem_bytes(dev_.h.nwords, npad_, maxGroup_, codeMode_);
}

bool Updater::residentEligible() const
{
    if (!initialized()) return false;
    return residentSmem() <= kResidentMaxSmem && maxGroup_ <= 16u * kResidentBlock;
}

// ============================================================================ run

StepEntry Updater::nextStep()
{
    uint32_t const nC = (uint32_t)grpSize_.size();
    uint32_t d0, d1;
    if (drawKind_ == kDrawCounter) {
        d0 = counter_draw(drawSeed_, 2 * subStep_);
        d1 = counter_draw(drawSeed_, 2 * subStep_ + 1);
    } else {
        d0 = drawFn_(drawCtx_);
        d1 = drawFn_(drawCtx_);
    }
    StepEntry e;
    e.color = d0 % nC;
    e.seed = d1;
    e.parity = (uint32_t)(subStep_ & 1u);
    e.prevColor = lastColor_;
    e.off = grpOff_[e.color];
    e.cnt = grpSize_[e.color];
    e.poff = lastColor_ == kNoColor ? 0u : grpOff_[lastColor_];
    e.pcnt = lastColor_ == kNoColor ? 0u : grpSize_[lastColor_];
    lastColor_ = e.color;
    ++subStep_;
    return e;
}

void Updater::fillSteps(uint32_t nSteps, StepEntry* buf, bool)
{
    for (uint32_t t = 0; t < nSteps; ++t) buf[t] = nextStep();
    chainValid_ = false;   // the host's entries go to the device's entry slots
}

void Updater::ensureStaging()
{
    // pinned staging of the step entries, allocated on the first run of this system's own paths
    // (systems advanced only by a Batch never need it)
    if (hSteps_) return;
    // one extra entry holds the copy of the persistent kernel's barrier state, and after it the
    // copy of the move counters
    static_assert(sizeof(GridSync) <= sizeof(StepEntry), "GridSync fits one staging entry");
    // (entry kStepCap), then the producer's state and the first entry of a chain (kStepCap + 1,
    // kStepCap + 2, copied together to the producer's slot and the first entry slot)
    void* p = nullptr;
    cuda_check(cudaHostAlloc(&p, sizeof(StepEntry) * (kStepCap + 3) + kStatBytes, cudaHostAllocMapped),
               "cudaHostAlloc(steps)");
    hSteps_ = static_cast<StepEntry*>(p);
    hStepCap_ = kStepCap;
    hGs_ = reinterpret_cast<GridSync*>(hSteps_ + kStepCap);
    std::memset(hGs_, 0, sizeof(GridSync));
    hGen_ = reinterpret_cast<StepGen*>(hSteps_ + kStepCap + 1);
    hStats_ = reinterpret_cast<unsigned long long*>(hSteps_ + kStepCap + 3);
    if (!genFree_) cuda_check(cudaEventCreateWithFlags(&genFree_, cudaEventDisableTiming), "cudaEventCreate");
    void* d = nullptr;
    cuda_check(cudaHostGetDevicePointer(&d, hStats_, 0), "stats staging device address");
    dStats_ = static_cast<unsigned long long*>(d);
}

void Updater::scrubPending(cudaStream_t s)
{
    if (lastColor_ == kNoColor) return;
    ensureStaging();
    // a perform launch with no current colour only zeroes the previous sub-step's marks
    cuda_check(cudaEventSynchronize(stepsFree_), "steps staging");
    hSteps_[0] = StepEntry{kNoColor, 0u, (uint32_t)(subStep_ & 1u), lastColor_, 0u, 0u, grpOff_[lastColor_],
                           grpSize_[lastColor_]};
    cuda_check(cudaMemcpyAsync(dev_.dSteps, hSteps_, sizeof(StepEntry), cudaMemcpyHostToDevice, s), "steps H2D");
    h2dBytes_ += sizeof(StepEntry);
    cuda_check(cudaEventRecord(stepsFree_, s), "event");
    chainValid_ = false;
    flushTickets();
    lastRunSnap_ = false;
    lastRunLead_ = false;
    // both representations scrub the previous sub-step's marks in the perform
    cuda_check(launchPerform(dev_.dSteps, s, performArgs(hSteps_[0])), "scrub");
    ++launches_;
    lastColor_ = kNoColor;
}

void Updater::noteExternalRun(uint64_t subSteps, uint64_t mcs, bool pendingMarks, uint32_t lastColor)
{
    (void)subSteps;
    lastRunSnap_ = false;
    lastRunLead_ = false;   // the batch flushed this system's waiting tickets before it ran
    mcsDone_ += mcs;
    hostStale_ = true;
    lastColor_ = pendingMarks ? lastColor : kNoColor;
}

void Updater::enqueueLaunch(uint32_t nSteps)
{
    for (uint32_t done = 0; done < nSteps;) {
        uint32_t const chunk = std::min(nSteps - done, hStepCap_);
        cuda_check(cudaEventSynchronize(stepsFree_), "steps staging");
        fillSteps(chunk, hSteps_, false);
        cuda_check(cudaMemcpyAsync(dev_.dSteps, hSteps_, sizeof(StepEntry) * chunk, cudaMemcpyHostToDevice, stream_),
                   "steps H2D");
        h2dBytes_ += sizeof(StepEntry) * chunk;
        cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        for (uint32_t t = 0; t < chunk; ++t) {
            cuda_check(launchCheck(dev_.dSteps + t, stream_), "check");
            cuda_check(launchPerform(dev_.dSteps + t, stream_, performArgs(hSteps_[t])), "perform");
        }
        launches_ += 2ull * chunk;
        done += chunk;
    }
}

cudaGraphExec_t Updater::graphFor(uint32_t nSteps, uint32_t parity0, bool snap)
{
    for (auto const& g : graphs_)
        if (g.nSteps == nSteps && g.parity0 == parity0 && g.snap == snap) return g.exec;
    // node t performs the sub-step whose entry sits in slot t and, in a graph of two or more
    // sub-steps, writes the entry of the next one into slot t + 1 (the last node into slot 0,
    // where the next replay starts) when the device producer is on; the perform's parity is a
    // launch parameter, so a graph is captured per length and parity of its first sub-step
    // snap: with bond codes the first check takes the counters' snapshot as the work before the
    // replay left them, on the gather representation a node after the last perform takes it
    bool const lead = snap && leadSnapshots();
    cudaGraph_t g;
    cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaSuccess;
    for (uint32_t t = 0; t < nSteps && err == cudaSuccess; ++t) {
        err = launchCheck(dev_.dSteps + t, stream_, lead && t == 0 ? dev_.snap : nullptr);
        PerformArgs pa;
        pa.parity = (parity0 + t) & 1u;
        pa.scope = kPerfCur | kPerfPrev;   // a scrub with no marks pending only zeroes zero words
        pa.next = nSteps >= 2 ? dev_.dSteps + (t + 1) % nSteps : nullptr;
        if (err == cudaSuccess) err = launchPerform(dev_.dSteps + t, stream_, pa);
    }
    if (snap && !lead && err == cudaSuccess)
        err = launch_snapshot_stats(dev_.h.stats, dev_.snap, dev_.snapSeq, stream_);
    cudaError_t const endErr = cudaStreamEndCapture(stream_, &g);
    cuda_check(err, "capture launches");
    cuda_check(endErr, "end capture");
    cudaGraphExec_t exec = nullptr;
    cudaError_t const instErr = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    cuda_check(instErr, "graph instantiate");
    graphs_.push_back({nSteps, parity0, snap, exec});
    return exec;
}

void Updater::prepareGraphs(uint32_t nSteps)
{
    // the (length, first parity) of every chunk a graph-path run of nSteps from here replays: the
    // full chunks start at no more than two parities, then the tail
    uint32_t const G = std::min(kGraphMcs * (uint32_t)grpSize_.size(), hStepCap_);
    uint32_t const full = nSteps / G, rest = nSteps % G;
    for (uint32_t k = 0; k < full && k < 2; ++k) graphFor(G, (uint32_t)((subStep_ + (uint64_t)k * G) & 1u), snapMode_);
    if (rest) graphFor(rest, (uint32_t)((subStep_ + (uint64_t)full * G) & 1u), snapMode_);
}

void Updater::seedChain(cudaStream_t s)
{
    // the first entry of a chain from the host, with the producer's state: one copy
    cuda_check(cudaEventSynchronize(genFree_), "producer staging");
    StepEntry const e0 = nextStep();
    hGen_[0] = StepGen{drawSeed_, subStep_, 1u, (uint32_t)grpSize_.size(), {0u, 0u}};
    std::memcpy(reinterpret_cast<StepEntry*>(hGen_) + 1, &e0, sizeof(StepEntry));
    cuda_check(cudaMemcpyAsync(dev_.h.gen, hGen_, 2 * sizeof(StepEntry), cudaMemcpyHostToDevice, s), "chain H2D");
    h2dBytes_ += 2 * sizeof(StepEntry);
    cuda_check(cudaEventRecord(genFree_, s), "event");
    genOn_ = 1;
}

void Updater::producerOff(cudaStream_t s)
{
    // host-made entries in the slots a captured graph reads: its nodes must not overwrite them
    if (genOn_ == 0) return;
    cuda_check(cudaEventSynchronize(genFree_), "producer staging");
    hGen_[0] = StepGen{0ull, 0ull, 0u, 0u, {0u, 0u}};
    cuda_check(cudaMemcpyAsync(dev_.h.gen, hGen_, sizeof(StepGen), cudaMemcpyHostToDevice, s), "producer off");
    h2dBytes_ += sizeof(StepGen);
    cuda_check(cudaEventRecord(genFree_, s), "event");
    genOn_ = 0;
}

void Updater::enqueueGraph(uint32_t nSteps)
{
    // full chunks of kGraphMcs MCS replay one graph; a shorter tail (or a short run) replays a
    // graph of its own length, captured once and kept. With the counter stream the device makes
    // the entries: the host copies only the first entry of a chain (and the producer's state)
    // when the device's chain does not continue from the host's position, otherwise nothing.
    uint32_t const nC = (uint32_t)grpSize_.size();
    uint32_t const G = std::min(kGraphMcs * nC, hStepCap_);
    bool const lead = snapMode_ && leadSnapshots();
    if (!lead) flushTickets();
    for (uint32_t done = 0; done < nSteps;) {
        uint32_t const chunk = std::min(G, nSteps - done);
        cudaGraphExec_t const exec = graphFor(chunk, (uint32_t)(subStep_ & 1u), snapMode_);
        if (drawKind_ == kDrawCounter && chunk >= 2) {
            uint32_t todo = chunk;
            if (!(chainValid_ && chainSub_ == subStep_ && chainPrev_ == lastColor_ && chainSeed_ == drawSeed_)) {
                seedChain(stream_);   // consumes the chunk's first sub-step
                --todo;
            }
            for (uint32_t t = 0; t < todo; ++t) nextStep();   // the host's copy of the position
            chainValid_ = true;
            chainSub_ = subStep_;
            chainPrev_ = lastColor_;
            chainSeed_ = drawSeed_;
        } else {
            producerOff(stream_);
            cuda_check(cudaEventSynchronize(stepsFree_), "steps staging");
            fillSteps(chunk, hSteps_, false);
            cuda_check(cudaMemcpyAsync(dev_.dSteps, hSteps_, sizeof(StepEntry) * chunk, cudaMemcpyHostToDevice,
                                       stream_),
                       "steps H2D");
            h2dBytes_ += sizeof(StepEntry) * chunk;
            cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        }
        cuda_check(cudaGraphLaunch(exec, stream_), "graph launch");
        launches_ += 2ull * chunk + (snapMode_ && !lead ? 1u : 0u);
        if (lead) publishPending(snapIssued_);   // this replay's first check wrote that snapshot
        if (snapMode_) ++snapIssued_;
        done += chunk;
    }
    lastRunSnap_ = snapMode_ && !lead;
    lastRunLead_ = lead;
}

float Updater::runTimed(int32_t nMcs)
{
    requireInit("runTimed");
    // a graph-path run of a new length captures its graphs first, outside the timed region (a
    // one-time host cost; the replays are what is timed)
    if (nMcs > 0 && (uint64_t)nMcs * grpSize_.size() <= 0xFFFFFFFFull) {
        cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
        ensureStaging();
        if (effectiveMode() == kModeGraph) prepareGraphs((uint32_t)nMcs * (uint32_t)grpSize_.size());
    }
    cudaEvent_t a, b;
    cuda_check(cudaEventCreate(&a), "cudaEventCreate");
    cuda_check(cudaEventCreate(&b), "cudaEventCreate");
    cuda_check(cudaEventRecord(a, stream_), "event");
    run(nMcs);
    cuda_check(cudaEventRecord(b, stream_), "event");
    cuda_check(cudaEventSynchronize(b), "timed run");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, a, b), "elapsed");
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

void Updater::timeKernels(int32_t nMcs, double out[4])
{
    // the grid-phase kernels one launch at a time, each bracketed by CUDA events on the stream
    // it runs on; sums per kernel
    requireInit("timeKernels");
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    flushTickets();
    lastRunSnap_ = false;
    lastRunLead_ = false;
    ensureStaging();
    scrubPending(stream_);
    uint32_t const nSteps = (uint32_t)nMcs * (uint32_t)grpSize_.size();
    std::vector<cudaEvent_t> ev(3);
    for (auto& e : ev) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
    double check = 0, perform = 0;
    uint64_t n = 0;
    for (uint32_t done = 0; done < nSteps;) {
        uint32_t const chunk = std::min(nSteps - done, hStepCap_);
        cuda_check(cudaEventSynchronize(stepsFree_), "steps staging");
        fillSteps(chunk, hSteps_, false);
        cuda_check(cudaMemcpyAsync(dev_.dSteps, hSteps_, sizeof(StepEntry) * chunk, cudaMemcpyHostToDevice, stream_),
                   "steps H2D");
        h2dBytes_ += sizeof(StepEntry) * chunk;
        cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        for (uint32_t t = 0; t < chunk; ++t) {
            cuda_check(cudaEventRecord(ev[0], stream_), "event");
            cuda_check(launchCheck(dev_.dSteps + t, stream_), "check");
            cuda_check(cudaEventRecord(ev[1], stream_), "event");
            cuda_check(launchPerform(dev_.dSteps + t, stream_, performArgs(hSteps_[t])), "perform");
            cuda_check(cudaEventRecord(ev[2], stream_), "event");
            cuda_check(cudaEventSynchronize(ev[2]), "timed kernels");
            float a = 0, b = 0;
            cuda_check(cudaEventElapsedTime(&a, ev[0], ev[1]), "elapsed");
            cuda_check(cudaEventElapsedTime(&b, ev[1], ev[2]), "elapsed");
            check += a;
            perform += b;
            ++n;
        }
        done += chunk;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    launches_ += 2 * n;
    mcsDone_ += (uint64_t)nMcs;
    hostStale_ = true;
    out[0] = check;
    out[1] = perform;
    out[2] = (double)n;
    out[3] = (double)n;
}

void Updater::enqueueResident(uint32_t nSteps)
{
    scrubPending(stream_);
    size_t const smem = residentSmem();
    uint32_t per = 1;
    while (per * kResidentBlock < maxGroup_) per *= 2;
    for (uint32_t done = 0; done < nSteps;) {
        uint32_t const chunk = std::min(nSteps - done, hStepCap_);
        cuda_check(cudaEventSynchronize(stepsFree_), "steps staging");
        fillSteps(chunk, hSteps_, true);
        cuda_check(cudaMemcpyAsync(dev_.dSteps, hSteps_, sizeof(StepEntry) * chunk, cudaMemcpyHostToDevice, stream_),
                   "steps H2D");
        h2dBytes_ += sizeof(StepEntry) * chunk;
        cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        cuda_check(codeMode_ == kCodeNone
                       ? launch_resident(dev_.dDesc, dev_.dList, 1, per, dev_.dSteps, 1, chunk, smem, stream_)
                       : launch_resident_bc(dev_.dDesc, dev_.dList, 1, per, dev_.dSteps, 1, chunk, smem, codeMode_,
                                            stream_),
                   "resident");
        ++launches_;
        done += chunk;
    }
    lastColor_ = kNoColor;   // the resident kernel leaves no marks in the global temporary lattices
}

void Updater::planCluster()
{
    // Tiers, each the smallest cluster (2..16 CTAs) the device can run whose CTAs walk at most so
    // many chunks of 32 slots per colour: 32 (one per warp) and then 48 (1.5 per warp), the plans
    // BFM_MODE_AUTO takes; 64 (2 per warp), the plan a Batch takes; 256 (8 per warp),
    // BFM_MODE_CLUSTER only. Each chunk a warp walks waits on remote shared memory, so the
    // kernel's time per sub-step grows with the chunks per warp more than with the cluster size.
    // Alone on a B200 (chains in 64^3 and 128^3 boxes, 11K-60K monomers, two barriers per
    // sub-step): one chunk per warp 8.9-11.3 us per MCS, up to 48 chunks per CTA 11.6-14.7, both
    // ahead of the persistent sweep (12.8-16.0); at 51-59 about even with it (15.3-16.9 against
    // 15.8) while still ahead of the graph of launches (17.9-18.1), the path a Batch runs such a
    // system on otherwise; at 8 chunks per warp 25-32.
    constexpr uint32_t kLimits[4] = {32u, 48u, 64u, 256u};
    constexpr uint32_t kTier[4] = {3u, 3u, 2u, 1u};
    clusterLogC_ = 0;
    clusterPer_ = 0;
    clusterSmem_ = 0;
    clusterTier_ = 0;
    if (codeMode_ == kCodeNone) return;
    uint32_t const chunks = (maxGroup_ + 31u) / 32u;
    for (uint32_t tier = 0; tier < 4; ++tier)
        for (uint32_t logC = 1; logC <= 4; ++logC) {
            uint32_t const C = 1u << logC;
            if (dev_.h.nwords < C) continue;
            uint32_t const perCta = (chunks + C - 1u) / C, perWarp = (perCta + 31u) / 32u;
            if (perCta > kLimits[tier]) continue;
            uint32_t per = 1;
            while (per < perWarp) per *= 2;
            size_t const smem = cluster_bc_smem_bytes(dev_.h.nwords, npad_, logC, per, codeMode_);
            if (smem > kResidentMaxSmem || !cluster_bc_runnable(logC, per, smem, codeMode_)) continue;
            clusterLogC_ = logC;
            clusterPer_ = per;
            clusterSmem_ = smem;
            clusterTier_ = kTier[tier];
            return;
        }
}

void Updater::enqueueCluster(uint32_t nSteps)
{
    scrubPending(stream_);
    for (uint32_t done = 0; done < nSteps;) {
        uint32_t const chunk = std::min(nSteps - done, hStepCap_);
        cuda_check(cudaEventSynchronize(stepsFree_), "steps staging");
        fillSteps(chunk, hSteps_, true);
        cuda_check(cudaMemcpyAsync(dev_.dSteps, hSteps_, sizeof(StepEntry) * chunk, cudaMemcpyHostToDevice, stream_),
                   "steps H2D");
        h2dBytes_ += sizeof(StepEntry) * chunk;
        cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        cuda_check(launch_cluster_bc(dev_.dDesc, dev_.dList, 1, clusterLogC_, clusterPer_, dev_.dSteps, 1, chunk,
                                     clusterSmem_, codeMode_, stream_),
                   "cluster");
        ++launches_;
        done += chunk;
    }
    lastColor_ = kNoColor;   // the cluster keeps its temporary lattice in shared memory
}

int Updater::path() const
{
    requireInit("path");
    return effectiveMode();
}

int Updater::autoMode() const
{
    // One system on a B200, per MCS: the resident kernel (one SM) while the largest colour group is
    // at most 2 x 1024 monomers (1.2K-3.3K-monomer chains 3.8-6.6 us, against 5.5-7.8 on a
    // cluster; 6.5K-8K: 11.4-13.2 against 8.3-8.8); then a cluster of CTAs holding the system in
    // distributed shared memory where each CTA walks at most 48 chunks of 32 slots per colour,
    // one per warp where a cluster of up to 16 CTAs allows (planCluster; 8K-47K monomers: 8.3-14.7
    // us against 12.8-16.0 persistent); then the
    // persistent sweep while its tiles fit about three per SM (to 262K monomers: 16-19 us against
    // 18-22 graph); beyond, the graph of separate launches (1M monomers: 30 us against 36).
    if (residentEligible() && maxGroup_ <= 2u * kResidentBlock) return kModeResident;
    if (clusterEligible() && clusterTier_ >= 3) return kModeCluster;
    if (codeMode_ != kCodeNone) {
        uint32_t const tiles = (maxGroup_ + kBcTileSpan - 1) / kBcTileSpan;
        if (tiles <= 3u * smCount_) return kModePersistent;
    }
    return kModeGraph;
}

int Updater::effectiveMode() const
{
    int m = mode_;
    if (m == kModeAuto) m = autoMode();
    if (m == kModeResident && !residentEligible()) m = kModeGraph;
    if (m == kModePersistent && codeMode_ == kCodeNone) m = kModeGraph;   // bond codes only
    if (m == kModeCluster && !clusterEligible()) m = kModeGraph;
    return m;
}

void Updater::run(int32_t nMcs)
{
    requireInit("runSimulationOnGPU");
    if (nMcs <= 0) return;
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    uint64_t const total = (uint64_t)nMcs * grpSize_.size();
    if (total > 0xFFFFFFFFull) throw std::invalid_argument("[runSimulationOnGPU] too many sub-steps in one call");
    uint32_t const nSteps = (uint32_t)total;
    ensureStaging();
    lastRunSnap_ = false;   // enqueueGraph sets both again
    lastRunLead_ = false;
    int const m = effectiveMode();
    if (m != kModeGraph) flushTickets();
    if (m == kModeResident) enqueueResident(nSteps);
    else if (m == kModeGraph) enqueueGraph(nSteps);
    else if (m == kModePersistent) enqueuePersistent(nSteps);
    else if (m == kModeCluster) enqueueCluster(nSteps);
    else enqueueLaunch(nSteps);
    mcsDone_ += (uint64_t)nMcs;
    hostStale_ = true;
}

namespace {
// CTAs per SM of the persistent kernel (launch_sweep_bc: 4, 5 or 6); 4, the default, is as fast
// as the others up to a few hundred thousand monomers and faster above. The environment variable
// BFM_SWEEP_SHAPE overrides it for tuning
int sweep_shape()
{
    static int const shape = [] {
        char const* e = std::getenv("BFM_SWEEP_SHAPE");
        int const v = e ? std::atoi(e) : 0;
        return (v >= 0 && v < kSweepShapes) ? v : 0;
    }();
    return shape;
}
}  // namespace

void Updater::enqueuePersistent(uint32_t nSteps)
{
    scrubPending(stream_);   // marks of a previous grid-phase run, left for the next check
    for (uint32_t done = 0; done < nSteps;) {
        uint32_t const chunk = std::min(nSteps - done, hStepCap_);
        cuda_check(cudaEventSynchronize(stepsFree_), "steps staging");
        fillSteps(chunk, hSteps_, false);
        cuda_check(cudaMemcpyAsync(dev_.dSteps, hSteps_, sizeof(StepEntry) * chunk, cudaMemcpyHostToDevice, stream_),
                   "steps H2D");
        h2dBytes_ += sizeof(StepEntry) * chunk;
        cuda_check(cudaEventRecord(stepsFree_, stream_), "event");
        // the arrival count restarts at 0 (an injected stall starts it at 0x80808080, from where no
        // barrier's target is reached); the fault word stays set once a launch has failed
        cuda_check(cudaMemsetAsync(&dev_.gs->count, stallNext_ ? 0x80 : 0, sizeof(unsigned int), stream_),
                   "clear grid barrier");
        // an injected stall tests the grid barrier in global memory, so that launch is cooperative
        bool const allowCluster = !stallNext_;
        stallNext_ = false;
        uint32_t grid = 0;
        cuda_check(launch_sweep_bc(dev_.h, dev_.dSteps, chunk, maxGroup_, dev_.gs, codeMode_, sweep_shape(),
                                   allowCluster, stream_, &grid),
                   "persistent sweep");
        ++launches_;
        done += chunk;
    }
    // the fault word comes back with the next synchronisation
    cuda_check(cudaMemcpyAsync(hGs_, dev_.gs, sizeof(GridSync), cudaMemcpyDeviceToHost, stream_), "grid status");
    d2hBytes_ += sizeof(GridSync);
    gsPending_ = true;
}

void Updater::runSimulationOnGPU(int32_t nMcs)
{
    run(nMcs);
    synchronize();
}

void Updater::streamWait(cudaEvent_t e)
{
    cuda_check(cudaStreamWaitEvent(stream_, e, 0), "cudaStreamWaitEvent");
}

void Updater::synchronize()
{
    if (stream_) cuda_check(cudaStreamSynchronize(stream_), "sweep");
    if (gsPending_) {
        gsPending_ = false;
        if (hGs_->fault) {
            std::ostringstream m;
            m << "[runSimulationOnGPU] a grid barrier of the persistent sweep timed out (barrier " << hGs_->where
              << "); the system's state is not usable";
            throw CudaError(m.str());
        }
    }
}

// ============================================================================ read back

void Updater::downloadPositions(int32_t* out)
{
    // the device puts the positions into the caller's order; one copy brings them over
    cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
    cuda_check(launch_gather_positions(dev_.h, dev_.slotOf, n_, dev_.xyzOut, stream_), "gather positions");
    cuda_check(cudaMemcpyAsync(out, dev_.xyzOut, 12ull * n_, cudaMemcpyDeviceToHost, stream_), "download positions");
    d2hBytes_ += 12ull * n_;
    synchronize();
}

void Updater::pullPositions()
{
    if (!hostStale_ || !initialized()) return;
    if (n_) downloadPositions(xyz_.data());
    hostStale_ = false;
}

int32_t Updater::getMonomerPosition(uint32_t i, int axis)
{
    requireN("getMonomerPosition");
    if (i >= n_ || axis < 0 || axis > 2) throw std::out_of_range("[getMonomerPosition] index out of range");
    pullPositions();
    return xyz_[3 * (size_t)i + axis];
}

void Updater::getCoordinates(int32_t* xyz, uint32_t n)
{
    requireN("getCoordinates");
    if (n != n_) throw std::invalid_argument("[getCoordinates] wrong monomer count");
    if (hostStale_ && initialized()) {
        // straight into the caller's buffer; the host copy stays stale until a getter needs it
        if (n_) downloadPositions(xyz);
        return;
    }
    std::memcpy(xyz, xyz_.data(), sizeof(int32_t) * 3 * (size_t)n_);
}

void Updater::setCoordinates(int32_t const* xyz, uint32_t n)
{
    requireN("setCoordinates");
    if (n != n_) throw std::invalid_argument("[setCoordinates] wrong monomer count");
    if (initialized())
        for (uint32_t i = 0; i < n_; ++i)
            for (int a = 0; a < 3; ++a)
                if (((walls_ >> a) & 1u) && uint32_t(xyz[3ull * i + a]) >= box_[a] - 1u)
                    throw std::invalid_argument("[setCoordinates] monomer " + std::to_string(i) +
                                                " lies outside the walls of the box");
    if (xyz != xyz_.data()) std::memcpy(xyz_.data(), xyz, sizeof(int32_t) * 3 * (size_t)n_);
    hostStale_ = false;
    if (!initialized()) return;
    // re-upload positions in sorted order and rebuild the occupancy lattice on the device
    synchronize();
    std::vector<int32_t> hx(npad_, kPadCoord), hy(npad_, 0), hz(npad_, 0);
    for (uint32_t i = 0; i < n_; ++i) {
        uint32_t const s = oldToNew_[i];
        hx[s] = xyz_[3 * (size_t)i];
        hy[s] = xyz_[3 * (size_t)i + 1];
        hz[s] = xyz_[3 * (size_t)i + 2];
    }
    scrubPending(stream_);
    cuda_check(cudaMemcpyAsync(dev_.h.x, hx.data(), 4ull * npad_, cudaMemcpyHostToDevice, stream_), "upload x");
    cuda_check(cudaMemcpyAsync(dev_.h.y, hy.data(), 4ull * npad_, cudaMemcpyHostToDevice, stream_), "upload y");
    cuda_check(cudaMemcpyAsync(dev_.h.z, hz.data(), 4ull * npad_, cudaMemcpyHostToDevice, stream_), "upload z");
    cuda_check(cudaMemsetAsync(dev_.h.lat, 0, 8ull * dev_.h.nwords, stream_), "clear lattice");
    cuda_check(launch_build_lattice(dev_.dDesc, npad_, stream_), "build lattice");
    std::vector<uint32_t> hpk, hnbrr;
    std::vector<uint8_t> hcode;
    std::vector<uint32_t> hrec;
    if (codeMode_ != kCodeNone) {
        hostCodes(hpk, hcode, hnbrr);
        hrec = slotRecords(hpk, hcode);
        cuda_check(cudaMemcpyAsync(dev_.h.rec, hrec.data(), 4ull * hrec.size(), cudaMemcpyHostToDevice, stream_),
                   "upload slot records");
        // the lattice above was built from the unfolded positions; bond codes keep image offsets
        toImageOffsets(hx, hy, hz);
        cuda_check(cudaMemcpyAsync(dev_.h.x, hx.data(), 4ull * npad_, cudaMemcpyHostToDevice, stream_), "upload x");
        cuda_check(cudaMemcpyAsync(dev_.h.y, hy.data(), 4ull * npad_, cudaMemcpyHostToDevice, stream_), "upload y");
        cuda_check(cudaMemcpyAsync(dev_.h.z, hz.data(), 4ull * npad_, cudaMemcpyHostToDevice, stream_), "upload z");
    }
    cuda_check(cudaStreamSynchronize(stream_), "setCoordinates");
}

uint32_t Updater::nColors() const
{
    requireInit("nColors");
    return (uint32_t)grpSize_.size();
}

std::vector<uint32_t> Updater::groupSizes() const
{
    requireInit("groupSizes");
    return grpSize_;
}

void Updater::stats(uint64_t out[4])
{
    requireInit("stats");
    // the sums written into the mapped pinned staging by a kernel on the stream
    ensureStaging();
    cuda_check(launch_publish_stats(dev_.h.stats, dStats_, stream_), "stats");
    d2hBytes_ += 3 * sizeof(unsigned long long);   // written into mapped host memory
    cuda_check(cudaStreamSynchronize(stream_), "stats");
    std::atomic_thread_fence(std::memory_order_acquire);
    unsigned long long const volatile* const sums = hStats_;
    for (uint32_t c = 0; c < 3; ++c) out[c] = sums[c];
    out[3] = mcsDone_;
}

uint64_t Updater::statsEnqueue()
{
    requireInit("stats");
    if (!hStatRing_) {
        void* p = nullptr;
        cuda_check(cudaHostAlloc(&p, 4 * sizeof(unsigned long long) * kStatRing, cudaHostAllocMapped),
                   "cudaHostAlloc(stats ring)");
        hStatRing_ = static_cast<unsigned long long*>(p);
        void* d = nullptr;
        cuda_check(cudaHostGetDevicePointer(&d, p, 0), "stats ring device address");
        dStatRing_ = static_cast<unsigned long long*>(d);
        for (cudaEvent_t& e : statEv_) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    }
    // the sums are written into host memory by a kernel (no copy-engine transfer between the
    // kernels); a slot's new write waits for its previous one, whichever stream made it
    uint64_t const t = ++statNext_;
    uint32_t const k = (uint32_t)(t % kStatRing);
    // a waiting ticket of this ring slot is older than the last kStatRing: it is dropped
    pendingTickets_.erase(std::remove(pendingTickets_.begin(), pendingTickets_.end(), k), pendingTickets_.end());
    if (lastRunLead_) {
        // the next replay's first check takes the snapshot of the counters as they are now
        pendingTickets_.push_back(k);
        statSeq_[k] = 0;
    } else if (lastRunSnap_) {
        // the last graph replay left its counters in snapshot slot (snapIssued_ - 1): copy that into
        // host memory on the publishing stream, so the sweep's stream goes on at once
        if (!pubStream_) {
            cuda_check(cudaStreamCreateWithFlags(&pubStream_, cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_check(cudaEventCreateWithFlags(&pubEv_, cudaEventDisableTiming), "cudaEventCreate");
        }
        cuda_check(cudaEventRecord(pubEv_, stream_), "event");
        cuda_check(cudaStreamWaitEvent(pubStream_, pubEv_, 0), "wait");
        cuda_check(cudaStreamWaitEvent(pubStream_, statEv_[k], 0), "wait");
        uint64_t const slot = (snapIssued_ - 1) % kSnapRing;
        cuda_check(launch_publish_snap(dev_.snap + 4 * slot, dStatRing_ + 4ull * k, pubStream_), "stats");
        cuda_check(cudaEventRecord(statEv_[k], pubStream_), "event");
        statSeq_[k] = snapIssued_;
    } else {
        cuda_check(cudaStreamWaitEvent(stream_, statEv_[k], 0), "wait");
        cuda_check(launch_publish_stats(dev_.h.stats, dStatRing_ + 4ull * k, stream_), "stats");
        cuda_check(cudaEventRecord(statEv_[k], stream_), "event");
        statSeq_[k] = 0;
        // this handle's counters are read by ticket: later graph-path runs end with a snapshot
        snapMode_ = true;
    }
    d2hBytes_ += 3 * sizeof(unsigned long long);   // written into mapped host memory
    statTicket_[k] = t;
    statMcs_[k] = mcsDone_;
    return t;
}

void Updater::publishPending(uint64_t snapSeq)
{
    // after the replay that writes snapshot snapSeq: the waiting tickets copy it on pubStream_
    if (pendingTickets_.empty()) return;
    if (!pubStream_) {
        cuda_check(cudaStreamCreateWithFlags(&pubStream_, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_check(cudaEventCreateWithFlags(&pubEv_, cudaEventDisableTiming), "cudaEventCreate");
    }
    cuda_check(cudaEventRecord(pubEv_, stream_), "event");
    cuda_check(cudaStreamWaitEvent(pubStream_, pubEv_, 0), "wait");
    uint64_t const slot = snapSeq % kSnapRing;
    for (uint32_t k : pendingTickets_) {
        cuda_check(cudaStreamWaitEvent(pubStream_, statEv_[k], 0), "wait");
        cuda_check(launch_publish_snap(dev_.snap + 4 * slot, dStatRing_ + 4ull * k, pubStream_), "stats");
        cuda_check(cudaEventRecord(statEv_[k], pubStream_), "event");
        statSeq_[k] = snapSeq + 1;
    }
    pendingTickets_.clear();
}

void Updater::flushTickets()
{
    // nothing has changed the counters since these tickets were taken: read them directly
    if (pendingTickets_.empty()) return;
    for (uint32_t k : pendingTickets_) {
        cuda_check(cudaStreamWaitEvent(stream_, statEv_[k], 0), "wait");
        cuda_check(launch_publish_stats(dev_.h.stats, dStatRing_ + 4ull * k, stream_), "stats");
        cuda_check(cudaEventRecord(statEv_[k], stream_), "event");
        statSeq_[k] = 0;
    }
    pendingTickets_.clear();
}

void Updater::statsWait(uint64_t ticket, uint64_t out[4])
{
    requireInit("stats");
    uint32_t const k = (uint32_t)(ticket % kStatRing);
    if (ticket == 0 || !hStatRing_ || statTicket_[k] != ticket)
        throw std::invalid_argument("[stats] unknown ticket, or one older than the last 8 of this system");
    if (std::find(pendingTickets_.begin(), pendingTickets_.end(), k) != pendingTickets_.end()) flushTickets();
    cuda_check(cudaEventSynchronize(statEv_[k]), "stats");
    std::atomic_thread_fence(std::memory_order_acquire);
    unsigned long long const volatile* const slot = hStatRing_ + 4ull * k;
    if (statSeq_[k] != 0 && slot[3] != statSeq_[k])
        throw CudaError("[stats] the counters' snapshot was replaced before it was copied (more than 64 graph "
                        "replays ahead of the read)");
    for (uint32_t c = 0; c < 3; ++c) out[c] = slot[c];
    out[3] = statMcs_[k];
}

void Updater::validate()
{
    // checkSystem, UpdaterGPUScBFM_AB_Type.cu:882-986: 8 cells per monomer without overlap, and
    // every bond in the allowed set (looked up with the kernel's 3-bit component index).
    requireN("validate");
    pullPositions();
    for (uint32_t i = 0; i < n_; ++i)
        for (int a = 0; a < 3; ++a)
            if (((walls_ >> a) & 1u) && uint32_t(xyz_[3ull * i + a]) >= box_[a] - 1u)
                throw std::runtime_error("[validate] monomer " + std::to_string(i) + " crossed a wall");
    // cells on the lattice (a walled axis of any side sits in a power-of-two lattice side and never
    // wraps; a periodic axis wraps with its mask)
    uint32_t const P[3] = {latticeSide(0), latticeSide(1), latticeSide(2)};
    uint64_t const V = (uint64_t)P[0] * P[1] * P[2];
    std::vector<uint8_t> cells(V, 0);
    uint64_t occupied = 0;
    for (uint32_t i = 0; i < n_; ++i)
        for (int c = 0; c < 8; ++c) {
            uint32_t const x = uint32_t(xyz_[3 * (size_t)i] + (c & 1)) & (P[0] - 1);
            uint32_t const y = uint32_t(xyz_[3 * (size_t)i + 1] + ((c >> 1) & 1)) & (P[1] - 1);
            uint32_t const z = uint32_t(xyz_[3 * (size_t)i + 2] + ((c >> 2) & 1)) & (P[2] - 1);
            uint8_t& cell = cells[x + (uint64_t)P[0] * (y + (uint64_t)P[1] * z)];
            occupied += cell ? 0 : 1;
            cell = 1;
        }
    if (occupied != 8ull * n_) {
        std::ostringstream m;
        m << "[checkSystem] Occupation count in the lattice is wrong! Expected 8*nMonomers=" << 8ull * n_
          << " occupied cells, but got " << occupied;
        throw std::runtime_error(m.str());
    }
    for (uint32_t i = 0; i < n_; ++i)
        for (uint32_t k = 0; k < nbrCnt_[i]; ++k) {
            uint32_t const j = nbrIds_[(size_t)i * kMaxConn + k];
            int32_t const dx = xyz_[3 * (size_t)j] - xyz_[3 * (size_t)i];
            int32_t const dy = xyz_[3 * (size_t)j + 1] - xyz_[3 * (size_t)i + 1];
            int32_t const dz = xyz_[3 * (size_t)j + 2] - xyz_[3 * (size_t)i + 2];
            uint32_t const idx = (uint32_t(dx) & 7u) | ((uint32_t(dy) & 7u) << 3) | ((uint32_t(dz) & 7u) << 6);
            if (forbidden_[idx]) {
                std::ostringstream m;
                m << "[checkSystem] This particular bond is forbidden: (" << dx << "," << dy << "," << dz
                  << ") between monomer " << i + 1 << " and monomer " << j + 1;
                throw std::runtime_error(m.str());
            }
        }
    // device-side consistency: the occupancy lattice, and in the bond-code representation the
    // packed coordinates and bond codes, must equal what the positions imply
    if (initialized()) {
        synchronize();
        std::vector<unsigned long long> lat(dev_.h.nwords);
        cuda_check(cudaMemcpy(lat.data(), dev_.h.lat, 8ull * lat.size(), cudaMemcpyDeviceToHost), "download lattice");
        std::vector<uint32_t> tab = brick_tables(dev_.h.nb);
        std::vector<unsigned long long> want(dev_.h.nwords, 0ull);
        for (uint32_t i = 0; i < n_; ++i) {
            uint32_t const mx = uint32_t(xyz_[3 * (size_t)i]) & dev_.h.mask[0];
            uint32_t const my = uint32_t(xyz_[3 * (size_t)i + 1]) & dev_.h.mask[1];
            uint32_t const mz = uint32_t(xyz_[3 * (size_t)i + 2]) & dev_.h.mask[2];
            uint32_t const w = tab[mx >> 2] + tab[dev_.h.nb[0] + (my >> 2)] + tab[dev_.h.nb[0] + dev_.h.nb[1] + (mz >> 2)];
            want[w] |= 1ull << (host_brick_pos(mx & 3, 0) | host_brick_pos(my & 3, 1) | host_brick_pos(mz & 3, 2));
        }
        if (lat != want) throw std::runtime_error("[checkSystem] device occupancy lattice disagrees with the positions");
        if (codeMode_ != kCodeNone) {
            std::vector<uint32_t> hpk, hnbrr;
            std::vector<uint8_t> hcode;
            hostCodes(hpk, hcode, hnbrr);
            std::vector<uint32_t> const want = slotRecords(hpk, hcode);
            std::vector<uint32_t> drec(want.size());
            cuda_check(cudaMemcpy(drec.data(), dev_.h.rec, 4ull * drec.size(), cudaMemcpyDeviceToHost),
                       "download slot records");
            uint32_t const rw = rec_words(codeMode_);
            for (uint32_t g = 0; g < npad_; ++g) {
                if (drec[(size_t)g * rw] != want[(size_t)g * rw])
                    throw std::runtime_error("[checkSystem] packed coordinates disagree with the positions");
                uint32_t const* const dc = drec.data() + (size_t)g * rw + rw / 2;
                if (!std::equal(dc, dc + rw / 2, want.data() + (size_t)g * rw + rw / 2))
                    throw std::runtime_error("[checkSystem] bond codes disagree with the positions");
            }
        }
    }
}

// ============================================================================ teardown

void Updater::freeDevice()
{
    // the publishing stream reads the arena's snapshots and writes the host ring: done first
    if (pubStream_) {
        cudaStreamSynchronize(pubStream_);
        cudaStreamDestroy(pubStream_);
        pubStream_ = nullptr;
    }
    if (pubEv_) {
        cudaEventDestroy(pubEv_);
        pubEv_ = nullptr;
    }
    if (!graphs_.empty() && stream_) cudaStreamSynchronize(stream_);   // no graph of ours in flight
    for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
    graphs_.clear();
    // stream-ordered frees: after this system's queued work (and whatever its stream waits on,
    // such as the end of a Batch run), without waiting on the host or for other streams
    if (dev_.arena) {
        cudaSetDevice(gpu_);
        cudaFreeAsync(dev_.arena, stream_);
    }
    dev_ = Device{};
    if (obsArena_) cudaFreeAsync(obsArena_, stream_);
    obsArena_ = nullptr;
    obs_ = ObsDev{};
    dObsOut_ = nullptr;
    nMol_ = 0;
    molSize_.clear();
    if (genFree_) {
        cudaEventSynchronize(genFree_);
        cudaEventDestroy(genFree_);
        genFree_ = nullptr;
    }
    chainValid_ = false;
    genOn_ = 0;
    if (hSteps_) {
        cudaFreeHost(hSteps_);
        hSteps_ = nullptr;
        hGs_ = nullptr;
        hGen_ = nullptr;
        hStats_ = nullptr;
        dStats_ = nullptr;
        gsPending_ = false;
        hStepCap_ = 0;
    }
    if (stepsFree_) {
        cudaEventDestroy(stepsFree_);
        stepsFree_ = nullptr;
    }
    if (hStatRing_) {
        for (cudaEvent_t& e : statEv_) {
            if (e) cudaEventSynchronize(e);
            if (e) cudaEventDestroy(e);
            e = nullptr;
        }
        cudaFreeHost(hStatRing_);
        hStatRing_ = nullptr;
        dStatRing_ = nullptr;
        for (uint32_t k = 0; k < kStatRing; ++k) statTicket_[k] = 0;
    }
    pendingTickets_.clear();

}

void Updater::cleanup()
{
    // UpdaterGPUScBFM_AB_Type.cu:995-1001 frees everything initialize and the setters allocated;
    // here the system returns to its freshly constructed state so the setter sequence can repeat.
    freeDevice();
    n_ = 0;
    nSet_ = false;
    xyz_.clear();
    attr_.clear();
    nbrCnt_.clear();
    nbrIds_.clear();
    colour_.clear();
    grpOff_.clear();
    grpSize_.clear();
    oldToNew_.clear();
    latticePopulated_ = false;
    subStep_ = mcsDone_ = 0;
    lastColor_ = kNoColor;
    hostStale_ = false;
}

}  // namespace bfm
