// host_api.cpp -- the C ABI of the B200 package and the level-stepping driver.
//
// The driver restates, with device launches instead of per-patch callbacks:
//   fclaw2d_advance_all_levels / advance_level   src/fclaw2d_advance.c:54-357
//   fclaw2d_update_single_step                   src/fclaw2d_update_single_step.c:73-103
//   fclaw2d_ghost_update (one process)           src/fclaw2d_ghost_fill.c:611-830
//   fclaw2d_time_sync / correct_coarse_cells     src/fclaw2d_time_sync.c:66-202
//   fclaw2d_timeinterp                           src/fclaw2d_timeinterp.c:29-57
//   fclaw2d_regrid / fclaw2d_initialize          src/fclaw2d_regrid.c:44-335, src/fclaw2d_initialize.c:75-250
// All patch data stays in device memory; the host touches it only to install
// initial data and at regrid (one flag per patch down, repopulation ops up).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <algorithm>
#include <string>
#include <vector>
#include <chrono>
#include "apps.hpp"
#include "fc2d_b200.h"
#include "host_forest.hpp"
#include "kernels.h"

using namespace fcb;

static double wall_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// A specialised kernel (spec = its limiter) applies to the second-order method with
// second-order transverse terms, that limiter on every one of 3 waves of 3 fields, no
// capacity, no aux and no cubed sphere.
static bool spec_applies(const Step2Variant& v, const fc2d_b200_options_t& o)
{
    if (v.spec == 0) return true;
    if (o.order[0] != 2 || o.order[1] != 2 || o.mcapa != 0 || o.maux != 0 || o.meqn != 3 || o.mwaves != 3 ||
        o.app == FC2D_B200_APP_SPHERE)
        return false;
    for (int w = 0; w < 3; w++)
        if (o.mthlim[w] != v.spec) return false;
    return true;
}

// Patch-to-CTA variants of the fused update compiled for one solver shape (first: default).
// Where a specialised kernel applies, only its variants are offered, so that every
// variant the autotuner may pick gives the same results.
static std::vector<const Step2Variant*> step2_variants(const fc2d_b200_options_t& o, int rp)
{
    using Table = const Step2Variant* (*)(int*);
    static const Table tables[] = {step2_table_f64_adv, step2_table_f64_sw, step2_table_f64_euler,
                                   step2_table_f32w_adv, step2_table_f32w_sw, step2_table_f32w_euler};
    std::vector<const Step2Variant*> out, spec;
    for (Table t : tables) {
        int n = 0;
        const Step2Variant* v = t(&n);
        for (int i = 0; i < n; i++)
            if (v[i].precision == o.precision && v[i].rp == rp && v[i].mx == o.mx && v[i].my == o.my &&
                v[i].mbc == o.mbc && spec_applies(v[i], o))
                (v[i].spec ? spec : out).push_back(&v[i]);
    }
    return spec.empty() ? out : spec;
}

static thread_local std::string g_err;
static int fail(int code, const std::string& msg) { g_err = msg; return code; }
#define CK(call)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
struct DevVec {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    ~DevVec() { if (p) cudaFree(p); }
    cudaError_t assign(const std::vector<T>& v, cudaStream_t st)
    {
        if (v.size() > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            cap = v.size() + v.size() / 2 + 16;
            cudaError_t e = cudaMalloc(&p, cap * sizeof(T));
            if (e != cudaSuccess) { cap = 0; return e; }
        }
        n = v.size();
        if (n) return cudaMemcpyAsync(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice, st);
        return cudaSuccess;
    }
};

// A typed range of a TableArena.
template <class T>
struct DevView {
    T* p = nullptr;
    size_t n = 0;
};

// The ghost-fill and time-sync tables of a forest: one device allocation filled from
// one pinned host buffer, so a regrid uploads them with one copy.  Both grow by a
// half beyond the largest forest seen and are reused from one regrid to the next.
struct TableArena {
    char* dev = nullptr;
    char* host = nullptr;
    size_t cap = 0, used = 0;
    cudaEvent_t copied = nullptr;    // the last upload's copy out of host is done
    ~TableArena()
    {
        if (copied) cudaEventDestroy(copied);
        if (dev) cudaFree(dev);
        if (host) cudaFreeHost(host);
    }
    // before the host buffer is written again: the last upload has left it
    cudaError_t wait_copied() { return copied ? cudaEventSynchronize(copied) : cudaSuccess; }
    cudaError_t mark_copied(cudaStream_t st)
    {
        if (!copied) {
            cudaError_t e = cudaEventCreateWithFlags(&copied, cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        return cudaEventRecord(copied, st);
    }
    cudaError_t reserve(size_t bytes)
    {
        if (bytes <= cap) return cudaSuccess;
        if (dev) cudaFree(dev);
        if (host) cudaFreeHost(host);
        dev = nullptr; host = nullptr; cap = 0;
        const size_t c = bytes + bytes / 2 + (1 << 20);
        cudaError_t e = cudaMalloc(&dev, c);
        if (e == cudaSuccess) e = cudaHostAlloc(&host, c, cudaHostAllocDefault);
        if (e != cudaSuccess) return e;
        cap = c;
        return cudaSuccess;
    }
    static size_t span(size_t bytes) { return (bytes + 255) & ~(size_t)255; }
    // place v at the next 256-byte boundary (copied by fill(), so v must live until then);
    // its device range
    template <class T>
    DevView<T> put(const std::vector<T>& v)
    {
        DevView<T> r;
        r.p = reinterpret_cast<T*>(dev + used);
        r.n = v.size();
        if (!v.empty()) pending.push_back({host + used, reinterpret_cast<const char*>(v.data()), v.size() * sizeof(T)});
        used += span(v.size() * sizeof(T));
        return r;
    }
    // the placed vectors into the host buffer, in pieces on the host worker threads
    void fill()
    {
        constexpr size_t PIECE = 256 << 10;
        std::vector<Piece> work;
        for (const Piece& p : pending)
            for (size_t o = 0; o < p.bytes; o += PIECE) work.push_back({p.dst + o, p.src + o, std::min(PIECE, p.bytes - o)});
        pending.clear();
        parallel_for((int)work.size(), [&](int k) { std::memcpy(work[k].dst, work[k].src, work[k].bytes); });
    }

private:
    struct Piece { char* dst; const char* src; size_t bytes; };
    std::vector<Piece> pending;
};

struct LevelRanges {
    int copy_off = 0, copy_n = 0, avg_off = 0, avg_n = 0, interp_off = 0, interp_n = 0, phys_off = 0, phys_n = 0;
    int ti_off = 0, ti_n = 0;
};

struct fc2d_b200_solver {
    fc2d_b200_options_t o;
    Dims d;
    Forest forest;
    Forest forest_next;          // a regrid's new forest, swapped with forest (both keep their buffers)
    cudaStream_t st = nullptr;
    double *q = nullptr, *qlast = nullptr, *qinterp = nullptr, *aux = nullptr, *regs = nullptr;
    PatchDesc* desc = nullptr;
    int cap = 0;                                   // patch capacity of the slabs
    // second set of slabs: regrid repopulates into it and swaps, so a regrid
    // allocates only when the forest outgrows the spare's capacity
    struct Spare { double *q = nullptr, *qlast = nullptr, *qinterp = nullptr, *aux = nullptr, *regs = nullptr;
                   double* area = nullptr; PatchDesc* desc = nullptr; int cap = 0; } spare;
    DevVec<int> flags_dev;                         // regrid tag flags
    bool has_inflow = false;                       // mthbc = 0 sides take bc_dev (app inflow state)
    double* bc_dev = nullptr;                      // 8 doubles
    unsigned long long* newton_hist = nullptr;     // 32 bins, exact Euler solver
    void* mlp_blob = nullptr;                      // p*-seed network (null: PVRS start)
    bool use_mlp = false;
    // batch of independent forests (instances); empty: one forest of the options
    std::vector<fc2d_b200_instance_t> insts;
    double* inst_dt_dev = nullptr;                 // coarse dt of each instance (device)
    double* inst_dt_host = nullptr;                // pinned staging copy
    int ncfl = 1;                                  // CFL maxima kept (one per instance)
    bool pending = false;                          // advance launched, not yet finished
    double pending_t = 0.0;
    // phys_ok[l]: the ghost cells of level l on physical faces hold physical-BC
    // values (set by a ghost update).  False after initialization: the reference
    // fills no ghost cells there by default (init_ghostcell = 0,
    // src/fclaw2d_initialize.c:140), so the first step sees qinit's ghost values.
    unsigned char phys_ok[64] = {};
    std::vector<const Step2Variant*> vars;         // compiled patch-to-CTA variants of this shape
    int var = 0;                                   // the one in use
    int var_lev[33];                               // per level (autotuned), -1: var
    // level updates issued back to back (a subcycled step starts every level whose
    // time has come, finest first, with nothing between them) touch disjoint
    // patches, so they go out as one launch over consecutive levels
    struct PendingUpdate { bool active = false; int lev_hi = 0, lev_lo = 0, p0 = 0, np = 0, slot = 0, var = 0; };
    PendingUpdate pend;
    // time interpolations of consecutive coarser levels, issued back to back after
    // an update, likewise share one launch (each level with its own alpha)
    struct PendingTimeInterp { bool active = false; int lev_lo = 0, lev_hi = 0; LevelAlpha alpha{}; };
    PendingTimeInterp pend_ti;
    // interp_chain[l]: no cell the interpolation into level l+1 reads (level-l cells
    // and their stencil neighbours) is written by the interpolation into level l, so
    // the two (issued finer first) may share a launch; computed per forest
    unsigned char interp_chain[34] = {};
    StepParams* tune_params = nullptr;             // autotuner: dt = 0 parameters (device)
    DevVec<RepopOp> repop_dev;                     // regrid repopulation ops
    DevVec<double> snap;                           // batch regrid: q of instances whose forest is unchanged
    DevVec<int> keep_dev;
    DevVec<int> aux_src_dev;                       // regrid: where each new patch's aux comes from
    DevVec<double> aux_staged_dev;                 // regrid: aux of new patches from the app's setaux
    TableArena arena;                              // the tables below, on the device
    DevView<FillOp> t_copy;                        // copy2ghost region ops
    DevView<FillOp> t_avg;                         // average2ghost region ops
    double* area = nullptr;                        // cubed sphere: cell areas per patch (Dims::narea per patch)
    bool sphere = false;                           // the cubed-sphere app (manifold, 6 blocks)
    SphereFlow flow{};                             // its rotation: psi = omega (axis . x)
    DevVec<MetricOp> metric_dev;
    DevVec<double> minmax_dev;
    DevView<InterpEnt> t_interp;
    DevView<PhysEnt> t_phys;
    DevView<int> t_ti;
    DevView<SyncOp> t_sync;
    Tables tables;                                 // host copy of the gather tables (buffers reused)
    TableWork table_work;
    std::vector<unsigned char> interp_written;     // interpolation-chain scratch, all zero between uses
    double regrid_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // fc2d_b200_last_regrid_stats
    // Time-sync register resets not yet applied, per level: bit t for face type t (see
    // StepParams::reg_reset).  Inside an advance a time sync's resets are left to the
    // next update of each level, which starts those faces' accumulation from zero; the
    // sync at the end of an advance applies them.
    int reg_pending[34] = {0};
    LevelRanges lr[33];
    unsigned long long* cfl_dev = nullptr;
    unsigned long long* cfl_host = nullptr;
    unsigned int* status_dev = nullptr;            // device status word (STATUS_* bits)
    unsigned int* status_host = nullptr;           // pinned copy read with the CFL
    double* mass_dev = nullptr;
    int mass_cap = 0;
    // one forest partitioned over ranks (fc2d_b200_set_partition); null: one rank
    struct PartState {
        fc2d_b200_comm_t comm{};
        PartitionPlan plan;
        DevVec<int> slots;                         // halo send slots, then halo recv slots
        size_t nsend = 0, nrecv = 0;
        double* buf = nullptr;                     // packed send segments, then recv segments
        size_t buf_cap = 0;
        bool graphs_before = true;
        bool failed = false;                       // an exchange inside an advance failed
    };
    std::unique_ptr<PartState> part;
    double* qsave = nullptr;                       // save_step copy of q
    size_t qsave_n = 0;                            // doubles it holds (0: nothing saved)
    size_t qsave_cap = 0;
    unsigned forest_gen = 0, qsave_gen = 0;        // forest installs so far; the one qsave belongs to
    unsigned char phys_ok_save[64] = {};
    double cell_updates = 0;
    double t_curr = 0;
    bool initialized = false;
    // single_step_update protocol
    int ss_level = -1, ss_count = 0;
    // host-data protocol: the caller's patch arrays of the level being buffered
    struct HostPatch { int slot; double* q; const double* aux; };
    std::vector<HostPatch> ss_host;
    double* ss_stage = nullptr;                    // pinned staging of one level's q
    size_t ss_stage_cap = 0;
    // timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    int ev_used = 0;
    std::vector<std::pair<int, double>> upd_launch_bytes;   // (event index, algorithmic bytes)
    double upd_ms = 0, upd_bytes = 0;
    int upd_launches = 0, total_launches = 0;
    std::vector<cudaEvent_t> user_ev;
    // the most recent advance: host time building its schedule (the first traversal),
    // and the span of its work on the stream (events before the first copy and after
    // the last launch), fc2d_b200_last_step_timing
    cudaEvent_t step_ev[2] = {nullptr, nullptr};
    double step_host_ms = 0, step_device_ms = 0;
    // per-launch update parameters in device memory (filled each advance)
    static constexpr int PCAP = 1 << 14;
    StepParams* params_dev = nullptr;
    StepParams* params_host = nullptr;
    int n_upd = 0;
    bool emit = true;                              // false: host traversal only (fill parameters)
    bool fill = true;                              // fill params_host / count statistics
    // CUDA graph of one fclaw2d_advance_all_levels for the current forest
    bool use_graphs = true;
    bool programmatic = true;                      // advance kernels with programmatic dependent launch
    cudaGraphExec_t graph_exec = nullptr;
    bool graph_stale = true;                       // the launches changed: update (or rebuild) before replay
    int graph_nupd = -1;
    int graph_builds = 0, graph_updates = 0;       // instantiations / in-place updates so far
};

// The launches of an advance changed (new forest, tables, variant, launch mode): the
// next advance captures them again and updates the executable graph in place when
// the new capture has the same shape, else instantiates a new one.
static void invalidate_graph(fc2d_b200_solver* s) { s->graph_stale = true; }
static void release_graph(fc2d_b200_solver* s)
{
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    s->graph_exec = nullptr;
    s->graph_stale = true;
    s->graph_nupd = -1;
}

const char* fc2d_b200_last_error(void) { return g_err.c_str(); }

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
static int alloc_slabs(fc2d_b200_solver* s, int np)
{
    const Dims& d = s->d;
    if (np <= s->cap && s->q) return 0;
    int cap = np + np / 2 + 16;                   // a growing forest reallocates rarely
    double *q, *ql, *qi = nullptr, *aux = nullptr, *regs, *area = nullptr;
    PatchDesc* desc;
    if (s->sphere) CK(cudaMalloc(&area, (size_t)cap * d.narea() * sizeof(double)));
    CK(cudaMalloc(&q, (size_t)cap * d.nq() * sizeof(double)));
    CK(cudaMalloc(&ql, (size_t)cap * d.nq() * sizeof(double)));
    if (s->o.subcycle) CK(cudaMalloc(&qi, (size_t)cap * d.nq() * sizeof(double)));
    if (d.maux > 0) CK(cudaMalloc(&aux, (size_t)cap * d.naux() * sizeof(double)));
    CK(cudaMalloc(&regs, (size_t)cap * d.nreg() * sizeof(double)));
    CK(cudaMalloc(&desc, (size_t)cap * sizeof(PatchDesc)));
    CK(cudaMemsetAsync(q, 0, (size_t)cap * d.nq() * sizeof(double), s->st));
    CK(cudaMemsetAsync(ql, 0, (size_t)cap * d.nq() * sizeof(double), s->st));
    if (qi) CK(cudaMemsetAsync(qi, 0, (size_t)cap * d.nq() * sizeof(double), s->st));
    CK(cudaMemsetAsync(regs, 0, (size_t)cap * d.nreg() * sizeof(double), s->st));
    if (s->q) {
        // caller copies what it needs before freeing; here the old slabs are released
        cudaFree(s->q); cudaFree(s->qlast); if (s->qinterp) cudaFree(s->qinterp);
        if (s->aux) cudaFree(s->aux); cudaFree(s->regs); cudaFree(s->desc);
        if (s->area) cudaFree(s->area);
    }
    s->q = q; s->qlast = ql; s->qinterp = qi; s->aux = aux; s->regs = regs; s->desc = desc; s->cap = cap;
    s->area = area;
    return 0;
}

static void free_spare(fc2d_b200_solver* s)
{
    auto& sp = s->spare;
    if (sp.q) cudaFree(sp.q);
    if (sp.qlast) cudaFree(sp.qlast);
    if (sp.qinterp) cudaFree(sp.qinterp);
    if (sp.aux) cudaFree(sp.aux);
    if (sp.regs) cudaFree(sp.regs);
    if (sp.desc) cudaFree(sp.desc);
    if (sp.area) cudaFree(sp.area);
    sp = fc2d_b200_solver::Spare{};
}

// Make the spare slabs hold np patches.  Contents are undefined: regrid's
// repopulation writes every array of every new patch.
static int ensure_spare(fc2d_b200_solver* s, int np)
{
    auto& sp = s->spare;
    if (sp.q && np <= sp.cap) return 0;
    free_spare(s);
    const Dims& d = s->d;
    // the spare and the current slabs swap at every regrid: the spare at least as large
    const int cap = std::max(np + np / 2 + 16, s->cap);
    CK(cudaMalloc(&sp.q, (size_t)cap * d.nq() * sizeof(double)));
    CK(cudaMalloc(&sp.qlast, (size_t)cap * d.nq() * sizeof(double)));
    if (s->o.subcycle) CK(cudaMalloc(&sp.qinterp, (size_t)cap * d.nq() * sizeof(double)));
    if (d.maux > 0) CK(cudaMalloc(&sp.aux, (size_t)cap * d.naux() * sizeof(double)));
    CK(cudaMalloc(&sp.regs, (size_t)cap * d.nreg() * sizeof(double)));
    CK(cudaMalloc(&sp.desc, (size_t)cap * sizeof(PatchDesc)));
    if (s->sphere) CK(cudaMalloc(&sp.area, (size_t)cap * d.narea() * sizeof(double)));
    sp.cap = cap;
    return 0;
}

static std::vector<PatchDesc> make_desc(const Forest& f)
{
    std::vector<PatchDesc> hd(f.np());
    for (int i = 0; i < f.np(); i++) {
        const PatchInfo& P = f.p[i];
        PatchDesc pd{};
        pd.xlower = P.xlower; pd.ylower = P.ylower; pd.dx = P.dx; pd.dy = P.dy;
        pd.level = P.level;
        pd.phys_mask = (P.phys[0] ? 1 : 0) | (P.phys[1] ? 2 : 0) | (P.phys[2] ? 4 : 0) | (P.phys[3] ? 8 : 0);
        int ft = 0;
        for (int k = 0; k < 4; k++) ft |= (P.face_type[k] & 3) << (2 * k);
        pd.face_type = ft;
        pd.flags = P.has_fine_nbr ? PATCH_HAS_FINE_NBR : 0;
        for (int k = 0; k < 4; k++)
            if (P.bcc3[k]) pd.flags |= PATCH_BCC3 << k;
        pd.inst = P.inst;
        pd.block = P.block;
        hd[i] = pd;
    }
    return hd;
}

static int upload_desc_and_tables(fc2d_b200_solver* s)
{
    const Forest& f = s->forest;
    const std::vector<PatchDesc> hd = make_desc(f);
    Tables& T = s->tables;
    {
        std::string err;
        const double t0 = wall_ms();
        if (!build_tables(f, s->o.mthbc, s->has_inflow, T, s->table_work, err)) return fail(FC2D_B200_EFOREST, err);
        s->regrid_ms[4] = wall_ms() - t0;
    }
    if (s->part) {
        // partitioned: a new plan for this forest; the ghost-fill stages write only the
        // ghost cells of owned and ring-1 patches, interpolation and the time sync only
        // those of owned patches
        auto& P = *s->part;
        make_partition(f, P.comm.rank, P.comm.size, P.plan);
        const std::vector<char>& fill = P.plan.fill;
        const std::vector<int>& own = P.plan.owner;
        const int me = P.comm.rank, nq = s->d.nq();
        // keep the entries that pass, level by level, and move the level offsets
        auto filter = [](auto& v, int* off, auto keep) {
            size_t n = 0;
            for (int l = 0; l < 33; l++) {
                const size_t a = off[l], b = off[l + 1];
                off[l] = (int)n;
                for (size_t k = a; k < b; k++)
                    if (keep(v[k])) v[n++] = v[k];
            }
            off[33] = (int)n;
            v.resize(n);
        };
        filter(T.copy, T.copy_off, [&](const FillOp& e) { return fill[e.dst] != 0; });
        filter(T.avg, T.avg_off, [&](const FillOp& e) { return fill[e.dst] != 0; });
        filter(T.phys, T.phys_off, [&](const PhysEnt& e) { return fill[e.dst / nq] != 0; });
        filter(T.interp, T.interp_off, [&](const InterpEnt& e) { return own[e.dst / nq] == me; });
        filter(T.ti, T.ti_off, [&](int p) { return fill[p] != 0; });
        for (int i = 0; i < f.np(); i++)          // the corrections of owned patches only
            if (own[i] != me)
                for (int k = 0; k < SYNC_SLOTS; k++) T.sync[(size_t)i * SYNC_SLOTS + k].kind = SYNC_NONE;
        // halo slot lists (send, then receive), uploaded once per forest
        std::vector<int> slots;
        for (const auto& v : P.plan.send) slots.insert(slots.end(), v.begin(), v.end());
        P.nsend = slots.size();
        for (const auto& v : P.plan.recv) slots.insert(slots.end(), v.begin(), v.end());
        P.nrecv = slots.size() - P.nsend;
        if (!slots.empty()) CK(P.slots.assign(slots, s->st));
    }
    for (int l = 0; l < 33; l++) {
        LevelRanges& r = s->lr[l];
        r = LevelRanges();
        r.copy_off = T.copy_off[l]; r.copy_n = T.copy_off[l + 1] - T.copy_off[l];
        r.avg_off = T.avg_off[l]; r.avg_n = T.avg_off[l + 1] - T.avg_off[l];
        r.interp_off = T.interp_off[l]; r.interp_n = T.interp_off[l + 1] - T.interp_off[l];
        r.phys_off = T.phys_off[l]; r.phys_n = T.phys_off[l + 1] - T.phys_off[l];
        r.ti_off = T.ti_off[l]; r.ti_n = T.ti_off[l + 1] - T.ti_off[l];
    }
    const std::vector<InterpEnt>& interp = T.interp;
    {
        TableArena& A = s->arena;
        auto sz = [](const auto& v) { return TableArena::span(v.size() * sizeof(v[0])); };
        CK(A.wait_copied());
        CK(A.reserve(sz(hd) + sz(T.copy) + sz(T.avg) + sz(T.interp) + sz(T.phys) + sz(T.ti) + sz(T.sync)));
        A.used = 0;
        const DevView<PatchDesc> dv = A.put(hd);       // staged here, then copied into the slab's descriptors
        s->t_copy = A.put(T.copy);
        s->t_avg = A.put(T.avg);
        s->t_interp = A.put(T.interp);
        s->t_phys = A.put(T.phys);
        s->t_ti = A.put(T.ti);
        s->t_sync = A.put(T.sync);
        A.fill();
        if (A.used) CK(cudaMemcpyAsync(A.dev, A.host, A.used, cudaMemcpyHostToDevice, s->st));
        if (dv.n) CK(cudaMemcpyAsync(s->desc, dv.p, dv.n * sizeof(PatchDesc), cudaMemcpyDeviceToDevice, s->st));
        CK(A.mark_copied(s->st));
    }
    {   // interpolation chains: reads of level l's entries against writes of level l-1's
        std::vector<unsigned char>& written = s->interp_written;
        if (written.size() < (size_t)f.np() * s->d.nq()) written.resize((size_t)f.np() * s->d.nq(), 0);
        const int nx = s->d.nx();
        for (int l = 0; l < 34; l++) s->interp_chain[l] = 0;
        for (int l = 1; l <= 32; l++) {
            const LevelRanges& lo = s->lr[l - 1];
            const LevelRanges& hi = s->lr[l];
            for (int k = 0; k < lo.interp_n; k++) written[interp[lo.interp_off + k].dst] = 1;
            bool clash = false;
            for (int k = 0; k < hi.interp_n && !clash; k++) {
                const long c = interp[hi.interp_off + k].src;
                for (long o : {0L, -1L, 1L, (long)-nx, (long)nx})
                    if (c + o >= 0 && c + o < (long)written.size() && written[c + o]) { clash = true; break; }
            }
            for (int k = 0; k < lo.interp_n; k++) written[interp[lo.interp_off + k].dst] = 0;
            s->interp_chain[l] = clash ? 0 : 1;
        }
    }
    // no wait here: the copies run in stream order ahead of every launch that reads the
    // tables, and the next upload waits for this one's copy before it refills the buffer
    return 0;
}

static cudaEvent_t next_event(fc2d_b200_solver* s)
{
    if (s->ev_used >= (int)s->ev_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        s->ev_pool.push_back(e);
    }
    return s->ev_pool[s->ev_used++];
}

// ---------------------------------------------------------------------------
// level operations
// ---------------------------------------------------------------------------
// Launch parameters of one level update.
static StepParams make_params(const fc2d_b200_solver* s, int level, double t, double dt)
{
    const Forest& f = s->forest;
    StepParams sp{};
    sp.order1 = s->o.order[0]; sp.order2 = s->o.order[1];
    for (int k = 0; k < 8; k++) sp.mthlim[k] = s->o.mthlim[k];
    sp.mcapa = s->o.mcapa;
    sp.store_flux = s->o.time_sync && s->o.flux_correction;
    sp.accumulate_waves = s->o.time_sync && s->o.fluctuation_correction;
    // save_current_step is only read by time interpolation of the coarser levels
    sp.save_last = (s->o.subcycle && level < f.maxlevel_present) ? 1 : 0;
    sp.app = s->o.app;
    // reflecting walls whose ghost cells mirror the interior (FP32-wave mass rule)
    sp.wall_faces = 0;
    if (level >= 0 && level < 64 && s->phys_ok[level])
        for (int f = 0; f < 4; f++)
            if (s->o.mthbc[f] == 3) sp.wall_faces |= 1 << f;
    sp.dt = dt; sp.t = t; sp.grav = s->o.grav;
    sp.dry_tolerance = s->o.pdata[31] > 0 ? s->o.pdata[31] : 1e-3;
    sp.vt = 0.0;
    sp.gamma = s->o.gamma;
    sp.newton_tol = s->o.newton_tol;
    sp.newton_hist = s->newton_hist;
    sp.mlp = s->use_mlp ? s->mlp_blob : nullptr;
    sp.inst_dt = s->insts.empty() ? nullptr : s->inst_dt_dev;
    sp.status = s->status_dev;
    sp.reg_reset = 0;
    if (s->o.app == FC2D_B200_APP_SWIRL && s->o.tperiod != 0.0) {
        const double pi = 4.0 * std::atan(1.0), pi2 = 2.0 * pi;
        sp.vt = std::cos(pi2 * (t + dt / 2.0) / s->o.tperiod);
    }
    return sp;
}

// Launch the pending group of time interpolations (levels lev_lo..lev_hi).
static void flush_timeinterp(fc2d_b200_solver* s)
{
    fc2d_b200_solver::PendingTimeInterp& g = s->pend_ti;
    if (!g.active) return;
    g.active = false;
    const int off = s->lr[g.lev_lo].ti_off, n = s->lr[g.lev_hi].ti_off + s->lr[g.lev_hi].ti_n - off;
    if (n <= 0) return;
    if (s->fill) s->total_launches++;
    if (s->emit) launch_timeinterp(s->d, s->q, s->qlast, s->qinterp, s->t_ti.p + off, n, s->desc, g.alpha, s->st);
}

static int flush_updates(fc2d_b200_solver* s);
// Launch whatever is pending, in issue order (a time-interpolation group always
// follows the update group it was issued after, which it flushed).
static int flush_pending(fc2d_b200_solver* s)
{
    int rc = flush_updates(s);
    flush_timeinterp(s);
    return rc;
}

// Launch the pending group of level updates (one launch, levels lev_lo..lev_hi).
static int flush_updates(fc2d_b200_solver* s)
{
    fc2d_b200_solver::PendingUpdate& g = s->pend;
    if (!g.active) return 0;
    g.active = false;
    if (s->fill) { s->upd_launches++; s->total_launches++; }
    if (!s->emit) return 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (s->timing) { e0 = next_event(s); e1 = next_event(s); CK(cudaEventRecord(e0, s->st)); }
    LevelGroup lg{};
    lg.nlev = g.lev_hi - g.lev_lo + 1;
    for (int i = 0; i < lg.nlev; i++)
        lg.start[i] = (s->part ? s->part->plan.own_lo[g.lev_lo + i] : s->forest.lev_off[g.lev_lo + i]) - g.p0;
    cudaError_t e = s->vars[g.var]->fn(s->q, s->qlast, s->aux, s->regs, s->desc, g.p0, g.np, s->params_dev + g.slot,
                                       lg, s->cfl_dev, s->st);
    if (e != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("step2 launch: ") + cudaGetErrorString(e));
    if (s->timing) {
        CK(cudaEventRecord(e1, s->st));
        const double cells = (double)g.np * s->d.mx * s->d.my;
        const double bytes = cells * 8.0 * (2.0 * s->d.meqn + s->d.maux);
        s->upd_launch_bytes.push_back({s->ev_used - 2, bytes});
    }
    return 0;
}

// One level update (clawpack46_update over the level's patches).  It joins the
// pending group when it is the next coarser level right after it (same variant,
// its parameter block the next slot); anything else launches the group first.
static int update_level(fc2d_b200_solver* s, int level, double t, double dt)
{
    const Forest& f = s->forest;
    if (level < 0 || level > 32) return 0;
    const int p0 = s->part ? s->part->plan.own_lo[level] : f.lev_off[level];
    const int np = (s->part ? s->part->plan.own_hi[level] : f.lev_off[level + 1]) - p0;
    if (np <= 0) return 0;
    if (s->vars.empty()) return fail(FC2D_B200_ESTATE, "no update kernel: register the application solver first");
    if (s->n_upd >= fc2d_b200_solver::PCAP) return fail(FC2D_B200_EINVAL, "too many level updates in one advance");
    flush_timeinterp(s);                              // it reads q of levels this update may write
    const int slot = s->n_upd++;
    if (s->fill) {
        StepParams& sp = s->params_host[slot];
        sp = make_params(s, level, t, dt);
        sp.reg_reset = s->reg_pending[level];      // resets a time sync left to this update
        s->reg_pending[level] = 0;
        s->cell_updates += (double)np * s->d.mx * s->d.my;
        if (s->emit)
            CK(cudaMemcpyAsync((void*)(s->params_dev + slot), &sp, sizeof(StepParams), cudaMemcpyHostToDevice, s->st));
    }
    const int v = s->var_lev[level] >= 0 ? s->var_lev[level] : s->var;
    fc2d_b200_solver::PendingUpdate& g = s->pend;
    if (g.active && level == g.lev_lo - 1 && v == g.var && slot == g.slot + (g.lev_hi - level) && p0 + np == g.p0) {
        g.lev_lo = level;
        g.p0 = p0;
        g.np += np;
        return 0;
    }
    int rc = flush_updates(s);
    if (rc) return rc;
    g.active = true;
    g.lev_hi = g.lev_lo = level;
    g.p0 = p0;
    g.np = np;
    g.slot = slot;
    g.var = v;
    return 0;
}

static double* tsdata(fc2d_b200_solver* s, int ti) { return ti ? s->qinterp : s->q; }

// Stage launches over a range of levels [a, b]: the per-level tables are laid
// out level after level, so a range is one contiguous slice.  Copy, average and
// physical-BC stages of different levels touch disjoint cells and read no cell
// the same stage writes, so a range is one launch; interpolation stays one
// launch per level (coarser levels overwrite ghost cells the finer level's
// interpolation reads first, as in the reference's max-to-min level loop).
static bool lrange(int& a, int& b)
{
    if (a < 0) a = 0;
    if (b > 32) b = 32;
    return a <= b;
}
// Stage ranges as table segments: levels [a, b] of q, and (c >= 0) level c of the
// time-interpolated copy.  A stage on q and the same stage on the copy write
// different arrays and neither reads what the other writes (the copy's stage
// reads the copy, or fine interiors of q, which no ghost-fill stage writes), so
// both go out in one launch.
template <class E>
static GatherSeg<E> seg(const E* table, int off, int n, double* dst, const double* src)
{
    return GatherSeg<E>{dst, src, table + off, n};
}
// average2ghost of coarse levels [a, b] and copy2ghost of levels [ca, cb] (with level c
// of the time-interpolated copy for both) in one launch: the two stages write disjoint
// ghost cells and read interior cells only, so their order does not matter
static void average_copy_range(fc2d_b200_solver* s, int a, int b, int ca, int cb, int c)
{
    GatherSeg<FillOp> a0{nullptr, nullptr, nullptr, 0}, a1 = a0, c0 = a0, c1 = a0;
    if (lrange(a, b)) {
        const int off = s->lr[a].avg_off, n = s->lr[b].avg_off + s->lr[b].avg_n - off;
        if (n > 0) a0 = seg(s->t_avg.p, off, n, s->q, s->q);
    }
    if (c >= 0 && c <= 32 && s->lr[c].avg_n > 0)
        a1 = seg(s->t_avg.p, s->lr[c].avg_off, s->lr[c].avg_n, s->qinterp, s->q);
    if (lrange(ca, cb)) {
        const int off = s->lr[ca].copy_off, n = s->lr[cb].copy_off + s->lr[cb].copy_n - off;
        if (n > 0) c0 = seg(s->t_copy.p, off, n, s->q, s->q);
    }
    if (c >= 0 && c <= 32 && s->lr[c].copy_n > 0)
        c1 = seg(s->t_copy.p, s->lr[c].copy_off, s->lr[c].copy_n, s->qinterp, s->qinterp);
    if (a0.n + a1.n + c0.n + c1.n <= 0) return;
    (void)flush_pending(s);
    if (s->fill) s->total_launches++;
    if (s->emit) launch_average_copy(s->d, a0, a1, c0, c1, s->area, s->st);
}
static void phys_range(fc2d_b200_solver* s, int a, int b, int c)
{
    GatherSeg<PhysEnt> s0{nullptr, nullptr, nullptr, 0}, s1 = s0;
    if (lrange(a, b)) {
        const int off = s->lr[a].phys_off, n = s->lr[b].phys_off + s->lr[b].phys_n - off;
        if (n > 0) s0 = seg(s->t_phys.p, off, n, s->q, s->q);
    }
    if (c >= 0 && c <= 32 && s->lr[c].phys_n > 0)
        s1 = seg(s->t_phys.p, s->lr[c].phys_off, s->lr[c].phys_n, s->qinterp, s->qinterp);
    if (s0.n + s1.n <= 0) return;
    (void)flush_pending(s);
    if (s->fill) s->total_launches++;
    if (s->emit) launch_phys(s->d, s0, s1, s->bc_dev, s->st);
}
// clawpack46 interpolate2ghost of levels hi, hi-1, ..., lo on q (finer levels first,
// one launch when each is chained to the next, interp_chain) and, when c >= 0 and
// chained too, of level c from the time-interpolated copy in the same launch.
// Returns whether level c went out.
static bool interp_run(fc2d_b200_solver* s, int lo, int hi, int c)
{
    GatherSeg<InterpEnt> s0{nullptr, nullptr, nullptr, 0}, s1 = s0;
    if (lo < 0) lo = 0;
    if (hi > 32) hi = 32;
    if (lo <= hi) {
        const int off = s->lr[lo].interp_off, n = s->lr[hi].interp_off + s->lr[hi].interp_n - off;
        if (n > 0) s0 = seg(s->t_interp.p, off, n, s->q, s->q);
    }
    if (c >= 0 && c <= 32 && s->lr[c].interp_n > 0)
        s1 = seg(s->t_interp.p, s->lr[c].interp_off, s->lr[c].interp_n, s->q, s->qinterp);
    if (s0.n + s1.n <= 0) return c >= 0;
    (void)flush_pending(s);
    if (s->fill) s->total_launches++;
    if (s->emit) launch_interp(s->d, s0, s1, s->st);
    return c >= 0;
}

static void interpolate_levels(fc2d_b200_solver* s, int mincoarse, int maxcoarse, int time_interp)
{
    const int c = time_interp ? mincoarse - 1 : -1;
    bool c_done = c < 0;
    int l = std::min(maxcoarse, 32);
    while (l >= mincoarse && l >= 0) {
        int lo = l;
        while (lo - 1 >= mincoarse && lo - 1 >= 0 && s->interp_chain[lo]) lo--;
        const bool with_c = !c_done && lo == mincoarse && c >= 0 && c <= 32 && s->interp_chain[mincoarse];
        if (interp_run(s, lo, l, with_c ? c : -1)) c_done = true;
        l = lo - 1;
    }
    if (!c_done) interp_run(s, 0, -1, c);
}

// Partitioned forest: send q, qlast and registers of this rank's patches in the
// other ranks' halos and receive theirs (full: every patch to every rank).  The
// solver's stream is idle while the caller's transport runs.
static int halo_exchange(fc2d_b200_solver* s, bool full)
{
    auto& P = *s->part;
    const PartitionPlan& pl = P.plan;
    const int me = P.comm.rank, np = s->forest.np();
    std::vector<int> peers;
    std::vector<size_t> ns, nr;
    const int* sl = nullptr;
    std::vector<int> all;
    size_t nsend = 0, nrecv = 0;
    if (full) {
        std::vector<int> own;
        std::vector<std::vector<int>> theirs(P.comm.size);
        for (int i = 0; i < np; i++) {
            if (pl.owner[i] == me) own.push_back(i);
            else theirs[pl.owner[i]].push_back(i);
        }
        for (int r = 0; r < P.comm.size; r++) {
            if (r == me) continue;
            peers.push_back(r);
            ns.push_back(own.size());
            all.insert(all.end(), own.begin(), own.end());
        }
        nsend = all.size();
        for (int r = 0; r < P.comm.size; r++) {
            if (r == me) continue;
            nr.push_back(theirs[r].size());
            all.insert(all.end(), theirs[r].begin(), theirs[r].end());
        }
        nrecv = all.size() - nsend;
    } else {
        peers = pl.peers;
        for (size_t k = 0; k < peers.size(); k++) { ns.push_back(pl.send[k].size()); nr.push_back(pl.recv[k].size()); }
        nsend = P.nsend; nrecv = P.nrecv;
        sl = P.slots.p;
    }
    if (peers.empty()) return 0;
    DevVec<int> tmp;
    if (full) {
        CK(tmp.assign(all, s->st));
        sl = tmp.p;
    }
    const size_t per = 2 * (size_t)s->d.nq() + s->d.nreg();
    const size_t need = (nsend + nrecv) * per;
    if (P.buf_cap < need) {
        if (P.buf) CK(cudaFree(P.buf));
        P.buf = nullptr;
        P.buf_cap = 0;
        CK(cudaMalloc(&P.buf, need * sizeof(double)));
        P.buf_cap = need;
    }
    launch_pack_patches(s->d, sl, (int)nsend, s->q, s->qlast, s->regs, P.buf, s->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->st));
    std::vector<void*> sp(peers.size()), rp(peers.size());
    std::vector<size_t> sb(peers.size()), rb(peers.size());
    size_t so = 0, ro = nsend;
    for (size_t k = 0; k < peers.size(); k++) {
        sp[k] = P.buf + so * per; sb[k] = ns[k] * per * sizeof(double); so += ns[k];
        rp[k] = P.buf + ro * per; rb[k] = nr[k] * per * sizeof(double); ro += nr[k];
    }
    if (P.comm.exchange(P.comm.user, (int)peers.size(), peers.data(), sp.data(), sb.data(), rp.data(), rb.data()))
        return fail(FC2D_B200_ECUDA, "the halo exchange callback failed");
    launch_unpack_patches(s->d, sl + nsend, (int)nrecv, s->q, s->qlast, s->regs, P.buf + nsend * per, s->st);
    CK(cudaGetLastError());
    if (full) CK(cudaStreamSynchronize(s->st));   // tmp's slots are freed on return
    return 0;
}

static void ghost_update(fc2d_b200_solver* s, int minlevel, int maxlevel, int time_interp)
{
    if (s->part && s->emit) {
        // the halo arrives before any stage reads it (the time-interpolated copies of
        // halo patches, still pending, are computed after it)
        if (flush_updates(s) || halo_exchange(s, false)) s->part->failed = true;
    }
    if (s->fill)
        for (int l = std::max(minlevel, 0); l <= std::min(maxlevel, 63); l++) s->phys_ok[l] = 1;
    const int mincoarse = minlevel, maxcoarse = maxlevel - 1;
    const int ti = time_interp ? mincoarse - 1 : -1;      // level of the time-interpolated copy
    average_copy_range(s, mincoarse, maxcoarse, minlevel, maxlevel, ti);
    phys_range(s, mincoarse, maxcoarse, ti);
    interpolate_levels(s, mincoarse, maxcoarse, time_interp);
    // the reference applies the physical BC to the fine levels [mincoarse+1, maxlevel],
    // then to every level [minlevel, maxlevel]; a physical-BC entry reads no cell any
    // physical-BC entry writes, so the second pass rewrites the first's values and one
    // pass over [minlevel, maxlevel] leaves the same fields
    phys_range(s, minlevel, maxlevel, ti);
}

// fclaw2d_time_sync(minlevel, maxlevel) as two launches: every correction of
// the synced levels (same-size and fine-to-coarse, grouped per patch), then
// every register reset.  Per level the reference runs samesize, reset, f2c,
// reset; the corrections of different levels touch disjoint cells and read only
// registers no earlier reset of the sync touches (f2c reads half-size faces of
// the coarse level and double-size faces of the fine level), so the merged
// order gives the same values.
// Reset rule of fclaw2d_time_sync(minlevel a, maxlevel maxl) for a patch of level L, by
// face type (k_reset_sync): same-size and physical faces always, faces with finer
// neighbours below maxl, faces with coarser neighbours when the coarser level is synced.
static int reset_mask(int L, int a, int maxl)
{
    int m = (1 << 0) | (1 << 2);
    if (L < maxl) m |= 1 << 1;
    if (L - 1 >= a && L - 1 < maxl) m |= 1 << 3;
    return m;
}

// defer: leave the register resets to the next update of each synced level (inside an
// advance: no register is read between a sync and that update but by that update)
static void time_sync(fc2d_b200_solver* s, int minlevel, int maxlevel, bool defer = false)
{
    (void)maxlevel;
    const int maxl = std::min(s->o.maxlevel, 32);
    int a = std::max(minlevel, 0);
    if (a > maxl) return;
    const int p0 = s->forest.lev_off[a], p1 = s->forest.lev_off[maxl + 1];
    if (p1 > p0) {   // samesize and f2c corrections, levels [a, maxl]
        (void)flush_pending(s);
        if (s->fill) s->total_launches++;
        if (s->emit) launch_sync(s->d, s->q, s->regs, s->desc, s->t_sync.p, p0, p1 - p0, s->st);
    }
    if (defer) {
        if (s->fill)
            for (int L = a; L <= maxl; L++) s->reg_pending[L] |= reset_mask(L, a, maxl);
        return;
    }
    // applied now: every reset of this sync, which covers any left pending since
    for (int L = a; L <= maxl; L++) s->reg_pending[L] &= ~reset_mask(L, a, maxl);
    if (p1 > p0) {
        (void)flush_pending(s);
        if (s->fill) s->total_launches++;
        if (s->emit) launch_reset_sync(s->d, s->regs, s->desc, p0, p1 - p0, a, maxl, s->st);
    }
}

static void timeinterp(fc2d_b200_solver* s, int level, double alpha)
{
    if (level < 0 || level > 31 || !s->lr[level].ti_n) return;
    (void)flush_updates(s);
    fc2d_b200_solver::PendingTimeInterp& g = s->pend_ti;
    if (g.active && level == g.lev_hi + 1) {        // the lists of consecutive levels are contiguous
        g.lev_hi = level;
        g.alpha.a[level] = alpha;
        return;
    }
    flush_timeinterp(s);
    g.active = true;
    g.lev_lo = g.lev_hi = level;
    g.alpha.a[level] = alpha;
}

struct Tsc { int last_step, step_inc, total_steps; double current_time, dt_step; };

static int advance_level(fc2d_b200_solver* s, Tsc* ts, int level, int curr_fine_step)
{
    int rc = update_level(s, level, ts[level].current_time, ts[level].dt_step);
    if (rc) return rc;
    ts[level].last_step += ts[level].step_inc;
    ts[level].current_time += ts[level].dt_step;
    if (level > s->forest.minlevel_present) {
        const int last_coarse_step = ts[level - 1].last_step;
        if (last_coarse_step == curr_fine_step) {
            rc = advance_level(s, ts, level - 1, last_coarse_step);
            if (rc) return rc;
            if (s->o.subcycle) {
                const int coarse_inc = ts[level - 1].step_inc;
                const int new_curr_step = ts[level].last_step;
                const double alpha = ((double)(new_curr_step % coarse_inc)) / coarse_inc;
                timeinterp(s, level - 1, alpha);
            }
        }
    }
    return 0;
}

static double bits_to_double(unsigned long long b)
{
    double v;
    std::memcpy(&v, &b, sizeof(v));
    return v;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
// Every entry point that touches the device makes the solver's device current for
// the call and puts the caller's device back on return.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(const fc2d_b200_solver* s);
    explicit DeviceScope(int device);
    ~DeviceScope() { if (prev >= 0) cudaSetDevice(prev); }
};

// ---------------------------------------------------------------------------
// Mass without device allocation: the scratch is the file-scope device array of
// k_mass_noalloc.cu, whose address is resolved once per device (with that
// device current) and cached.
// ---------------------------------------------------------------------------
static_assert(MASS_SCRATCH_DOUBLES == FC2D_B200_MASS_SCRATCH_DOUBLES,
              "the public scratch limit must equal the size of the device array");
static std::mutex g_scratch_mu;
static double* g_scratch_addr[128];

static int scratch_for_device(int dev, double** out)
{
    if (dev < 0 || dev >= 128) return fail(FC2D_B200_EINVAL, "device ordinal out of range for the mass scratch");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        int cur = -1;
        CK(cudaGetDevice(&cur));
        if (cur != dev) CK(cudaSetDevice(dev));
        double* p = nullptr;
        cudaError_t e = mass_scratch_address(&p);
        if (cur != dev) cudaSetDevice(cur);
        if (e != cudaSuccess || !p)
            return fail(FC2D_B200_ECUDA, std::string("cudaGetSymbolAddress(mass scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return 0;
}

DeviceScope::DeviceScope(int device)
{
    int cur = -1;
    if (device >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != device && cudaSetDevice(device) == cudaSuccess)
        prev = cur;
}
DeviceScope::DeviceScope(const fc2d_b200_solver* s) : DeviceScope(s ? s->o.device : -1) {}

extern "C" int fc2d_b200_create(const fc2d_b200_options_t* opt, fc2d_b200_solver_t** out)
{
    if (!opt || !out) return fail(FC2D_B200_EINVAL, "null argument");
    const fc2d_b200_options_t& o = *opt;
    if (o.mx <= 0 || o.my <= 0 || o.mbc < 2 || o.meqn <= 0 || o.meqn > 8 || o.maux < 0 || o.mwaves <= 0)
        return fail(FC2D_B200_EINVAL, "bad patch dimensions (need mx,my>0, mbc>=2, 0<meqn<=8)");
    if ((o.mx % 2) || (o.my % 2)) return fail(FC2D_B200_EINVAL, "mx and my must be even");
    if (o.time_sync && o.rp == FC2D_B200_RP_ADVECTION)
        return fail(FC2D_B200_EINVAL, "time sync needs a flux function (rpn2_cons): shallow water or Euler");
    if (o.rp == FC2D_B200_RP_EULER_EXACT && (o.meqn != 4 || o.mwaves != 3 || !(o.gamma > 1.0) || !(o.newton_tol > 0.0)))
        return fail(FC2D_B200_EINVAL, "exact Euler solver needs meqn 4, mwaves 3, gamma > 1, newton_tol > 0");
    if (o.minlevel < 0 || o.maxlevel < o.minlevel || o.maxlevel > 20)
        return fail(FC2D_B200_EINVAL, "bad minlevel/maxlevel");
    const bool user = o.rp == FC2D_B200_RP_USER;
    const bool sup = user || !step2_variants(o, o.rp).empty();
    if (!sup) return fail(FC2D_B200_EINVAL, "no compiled update kernel for this (rp, mx, my, mbc, precision)");
    if (user && (o.precision != FC2D_B200_PREC_FP64 || o.time_sync || o.mx != o.my || o.mbc != 2))
        return fail(FC2D_B200_EINVAL, "application solvers run in FP64, without time sync, on square patches with mbc 2");
    if (o.app == FC2D_B200_APP_SPHERE &&
        (o.rp != FC2D_B200_RP_ADVECTION_MANIFOLD || o.maux != 3 || o.mcapa != 1 || o.mx != o.my || o.mx < 8))
        return fail(FC2D_B200_EINVAL, "the cubed-sphere app needs the manifold advection solver, maux 3, mcapa 1, "
                                      "square patches with mx >= 8");
    if (o.app == FC2D_B200_APP_SPHERE && o.time_sync)
        return fail(FC2D_B200_EINVAL, "time sync across cubed-sphere block seams is not built");
    if (o.refinement_criteria < FC2D_B200_TAG_APP || o.refinement_criteria > FC2D_B200_TAG_GRADIENT_DX)
        return fail(FC2D_B200_EINVAL, "refinement_criteria must be one of FC2D_B200_TAG_*");
    if (o.threshold_variable < 0 || o.threshold_variable > o.meqn)
        return fail(FC2D_B200_EINVAL, "threshold_variable must be in 1..meqn (0: field 1)");
    if (o.smooth_level < 0) return fail(FC2D_B200_EINVAL, "smooth_level must be >= 0");
    if (o.regrid_interval < 0 || o.nout < 0) return fail(FC2D_B200_EINVAL, "regrid_interval and nout must be >= 0");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (ndev <= 0) return fail(FC2D_B200_ECUDA, "no CUDA device");
    if (o.device < 0 || o.device >= ndev) return fail(FC2D_B200_EINVAL, "device ordinal out of range");
    CK(cudaSetDevice(o.device));
    {   // load the allocation-free mass module and resolve its scratch now, outside any
        // step or stream capture (module loading is lazy and may allocate)
        double* scratch = nullptr;
        int rc = scratch_for_device(o.device, &scratch);
        if (rc) return rc;
    }
    auto s = std::make_unique<fc2d_b200_solver>();
    s->o = o;
    if (s->o.mi <= 0) s->o.mi = 1;
    if (s->o.mj <= 0) s->o.mj = 1;
    s->d = Dims{o.mx, o.my, o.mbc, o.meqn, o.maux};
    s->forest.g = Geometry{s->d, s->o.mi, s->o.mj, o.ax, o.bx, o.ay, o.by};
    if (o.app == FC2D_B200_APP_SPHERE) {
        // six blocks [0,1]^2, patch x coordinate = block 2^l + ix
        s->sphere = true;
        s->o.mi = 6; s->o.mj = 1; s->o.ax = 0.0; s->o.bx = 1.0; s->o.ay = 0.0; s->o.by = 1.0;
        s->forest.g = Geometry{s->d, 6, 1, 0.0, 1.0, 0.0, 1.0};
        s->forest.g.kind = 1;
        app_sphere_flow(s->o, s->flow.axis, &s->flow.omega);
    }
    CK(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
    CK(cudaMalloc(&s->cfl_dev, sizeof(unsigned long long) * FC2D_B200_MAX_INSTANCES));
    CK(cudaMallocHost(&s->cfl_host, sizeof(unsigned long long) * FC2D_B200_MAX_INSTANCES));
    CK(cudaMalloc(&s->status_dev, sizeof(unsigned int)));
    CK(cudaMemset(s->status_dev, 0, sizeof(unsigned int)));
    CK(cudaMallocHost(&s->status_host, sizeof(unsigned int)));
    CK(cudaMalloc(&s->inst_dt_dev, sizeof(double) * FC2D_B200_MAX_INSTANCES));
    CK(cudaMallocHost(&s->inst_dt_host, sizeof(double) * FC2D_B200_MAX_INSTANCES));
    CK(cudaMalloc(&s->params_dev, sizeof(StepParams) * fc2d_b200_solver::PCAP));
    {
        double bc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        s->has_inflow = app_inflow_state(s->o, bc);
        CK(cudaMalloc(&s->bc_dev, sizeof(bc)));
        CK(cudaMemcpy(s->bc_dev, bc, sizeof(bc), cudaMemcpyHostToDevice));
        CK(cudaMalloc(&s->newton_hist, 32 * sizeof(unsigned long long)));
        CK(cudaMemset(s->newton_hist, 0, 32 * sizeof(unsigned long long)));
    }
    CK(cudaMallocHost(&s->params_host, sizeof(StepParams) * fc2d_b200_solver::PCAP));
    {   // set the kernel's shared-memory attribute outside any stream capture
        s->vars = step2_variants(o, o.rp);
        s->var = 0;
        for (int l = 0; l < 33; l++) s->var_lev[l] = -1;
        if (!s->vars.empty()) {   // application solvers arrive with fc2d_b200_set_user_variants
            cudaError_t e = s->vars[0]->fn(nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0, nullptr, LevelGroup{1, {0}}, nullptr, s->st);
            if (e != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("kernel setup: ") + cudaGetErrorString(e));
        }
        CK(cudaMalloc(&s->tune_params, sizeof(StepParams)));
    }
    *out = s.release();
    return 0;
}

extern "C" int fc2d_b200_destroy(fc2d_b200_solver_t* s)
{
    DeviceScope dev_scope_(s);
    if (!s) return 0;
    cudaStreamSynchronize(s->st);
    for (auto e : s->ev_pool) cudaEventDestroy(e);
    for (auto e : s->user_ev) cudaEventDestroy(e);
    for (auto e : s->step_ev) if (e) cudaEventDestroy(e);
    cudaFree(s->q); cudaFree(s->qlast); if (s->qinterp) cudaFree(s->qinterp);
    if (s->aux) cudaFree(s->aux); cudaFree(s->regs); cudaFree(s->desc);
    free_spare(s);
    cudaFree(s->cfl_dev); cudaFreeHost(s->cfl_host); cudaFree(s->inst_dt_dev); cudaFreeHost(s->inst_dt_host);
    cudaFree(s->status_dev); cudaFreeHost(s->status_host);
    release_graph(s);
    cudaFree(s->params_dev); cudaFreeHost(s->params_host);
    if (s->mass_dev) cudaFree(s->mass_dev);
    if (s->qsave) cudaFree(s->qsave);
    if (s->ss_stage) cudaFreeHost(s->ss_stage);
    if (s->part && s->part->buf) cudaFree(s->part->buf);
    cudaFree(s->bc_dev); cudaFree(s->newton_hist);
    if (s->tune_params) cudaFree(s->tune_params);
    if (s->area) cudaFree(s->area);
    if (s->mlp_blob) cudaFree(s->mlp_blob);
    cudaStreamDestroy(s->st);
    delete s;
    return 0;
}

extern "C" int fc2d_b200_set_riemann(fc2d_b200_solver_t* s, int rp_id)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    std::vector<const Step2Variant*> vars = step2_variants(s->o, rp_id);
    if (vars.empty()) return fail(FC2D_B200_EINVAL, "Riemann solver id not compiled for these patch dimensions");
    s->o.rp = rp_id;
    s->vars = vars;
    s->var = 0;
    for (int l = 0; l < 33; l++) s->var_lev[l] = -1;
    invalidate_graph(s);
    cudaError_t e = s->vars[0]->fn(nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0, nullptr, LevelGroup{1, {0}}, nullptr, s->st);
    if (e != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("kernel setup: ") + cudaGetErrorString(e));
    return 0;
}

extern "C" int fc2d_b200_set_user_variants(fc2d_b200_solver_t* s, const void* table, int n, int abi, int meqn,
                                           int mwaves, int maux)
{
    DeviceScope dev_scope_(s);
    if (!s || !table || n <= 0) return fail(FC2D_B200_EINVAL, "null solver or empty variant table");
    if (abi != device_abi())
        return fail(FC2D_B200_EINVAL, "the application was built against another version of the kernel headers");
    if (s->o.rp != FC2D_B200_RP_USER) return fail(FC2D_B200_EINVAL, "the solver was not created with rp = FC2D_B200_RP_USER");
    if (meqn != s->o.meqn || mwaves != s->o.mwaves || maux != s->o.maux)
        return fail(FC2D_B200_EINVAL, "meqn / mwaves / maux of the application solver differ from the options");
    const Step2Variant* v = static_cast<const Step2Variant*>(table);
    std::vector<const Step2Variant*> vars;
    for (int i = 0; i < n; i++) {
        if (v[i].precision != FC2D_B200_PREC_FP64 || v[i].rp != FC2D_B200_RP_USER || v[i].mx != s->o.mx ||
            v[i].my != s->o.my || v[i].mbc != s->o.mbc || !v[i].fn)
            return fail(FC2D_B200_EINVAL, "variant " + std::to_string(i) + " does not fit the solver's patch shape");
        vars.push_back(&v[i]);
    }
    cudaError_t e = vars[0]->fn(nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0, nullptr, LevelGroup{1, {0}}, nullptr, s->st);
    if (e != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("kernel setup: ") + cudaGetErrorString(e));
    s->vars = vars;
    s->var = 0;
    for (int l = 0; l < 33; l++) s->var_lev[l] = -1;
    invalidate_graph(s);
    return 0;
}

// Install a new forest: slabs sized, descriptors and tables uploaded; data zero.
static int install_forest(fc2d_b200_solver* s, const std::vector<Leaf>& leaves)
{
    invalidate_graph(s);
    std::string err;
    Forest nf;
    nf.g = s->forest.g;
    nf.inst = s->forest.inst;
    if (!nf.build(leaves, err)) return fail(FC2D_B200_EFOREST, err);
    s->forest = std::move(nf);
    s->forest_gen++;
    std::memset(s->phys_ok, 0, sizeof(s->phys_ok));
    int rc = alloc_slabs(s, s->forest.np());
    if (rc) return rc;
    return upload_desc_and_tables(s);
}

extern "C" int fc2d_b200_set_forest(fc2d_b200_solver_t* s, int np, const int* level, const int* gx, const int* gy)
{
    DeviceScope dev_scope_(s);
    if (!s || np <= 0 || !level || !gx || !gy) return fail(FC2D_B200_EINVAL, "bad forest arguments");
    std::vector<Leaf> L(np);
    for (int i = 0; i < np; i++) L[i] = {level[i], gx[i], gy[i]};
    int rc = install_forest(s, L);
    if (rc) return rc;
    s->initialized = true;
    return 0;
}

// Options of instance i (a batch) or the solver's own.
static fc2d_b200_options_t inst_options(const fc2d_b200_solver* s, int i)
{
    fc2d_b200_options_t o = s->o;
    if (s->insts.empty()) return o;
    const fc2d_b200_instance_t& I = s->insts[i];
    o.minlevel = I.minlevel; o.maxlevel = I.maxlevel;
    o.ax = I.ax; o.bx = I.bx; o.ay = I.ay; o.by = I.by; o.mi = I.mi; o.mj = I.mj;
    for (int k = 0; k < 32; k++) o.pdata[k] = I.pdata[k];
    return o;
}
// Forest-level bounds of an instance (levels are relative to the instance's minlevel in a batch).
static int inst_minlev(const fc2d_b200_solver* s, int i) { (void)i; return s->insts.empty() ? s->o.minlevel : 0; }
static int inst_maxlev(const fc2d_b200_solver* s, int i)
{
    return s->insts.empty() ? s->o.maxlevel : s->insts[i].maxlevel - s->insts[i].minlevel;
}

extern "C" int fc2d_b200_initialize(fc2d_b200_solver_t* s)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    if (s->o.app == FC2D_B200_APP_NONE) return fail(FC2D_B200_EINVAL, "initialize needs a built-in app");
    const Dims& d = s->d;
    const int ni = s->forest.ninst();
    std::vector<fc2d_b200_options_t> io(ni);
    for (int i = 0; i < ni; i++) io[i] = inst_options(s, i);
    std::vector<Leaf> leaves;
    for (int i = 0; i < ni; i++) {
        const int l0 = inst_minlev(s, i), la = l0 + s->forest.gi(i).lbase;
        for (int y = 0; y < (io[i].mj << la); y++)
            for (int x = 0; x < (io[i].mi << la); x++) leaves.push_back({l0, x, y, i});
    }
    std::string err;
    Forest f;
    f.g = s->forest.g;
    f.inst = s->forest.inst;
    if (!f.build(leaves, err)) return fail(FC2D_B200_EFOREST, err);
    std::vector<double> q((size_t)f.np() * d.nq(), 0.0), aux((size_t)f.np() * d.naux(), 0.0);
    for (int i = 0; i < f.np(); i++) {
        const fc2d_b200_options_t& oi = io[f.p[i].inst];
        if (d.maux > 0) app_setaux(oi, d, f.p[i], &aux[(size_t)i * d.naux()]);
        app_qinit(oi, d, f.p[i], d.maux > 0 ? &aux[(size_t)i * d.naux()] : nullptr, &q[(size_t)i * d.nq()]);
    }
    // initial refinement (fclaw2d_initialize.c:150-230): tag with init_flag, new patches get qinit
    int maxspan = 0;
    for (int i = 0; i < ni; i++) maxspan = std::max(maxspan, inst_maxlev(s, i) - inst_minlev(s, i));
    for (int pass = 0; pass <= maxspan; pass++) {
        std::vector<int> mark(f.np(), 0);
        for (int i = 0; i < f.np(); i++) {
            const PatchInfo& P = f.p[i];
            if (P.level < inst_maxlev(s, P.inst) && app_tag_refine(io[P.inst], d, P, &q[(size_t)i * d.nq()])) mark[i] = 1;
        }
        if (s->o.smooth_refine) smooth_marks(f, mark, s->o.smooth_level);
        int changed = 0;
        std::vector<Leaf> L = adapt_leaves(f, mark, changed, err);
        if (!changed) break;
        Forest nf;
        nf.g = f.g;
        nf.inst = f.inst;
        if (!nf.build(L, err)) return fail(FC2D_B200_EFOREST, err);
        std::vector<double> nq((size_t)nf.np() * d.nq(), 0.0), naux((size_t)nf.np() * d.naux(), 0.0);
        for (int i = 0; i < nf.np(); i++) {
            const PatchInfo& P = nf.p[i];
            const int old = f.lookup(P.inst, P.level, P.gx, P.gy);
            if (old >= 0) {
                std::memcpy(&nq[(size_t)i * d.nq()], &q[(size_t)old * d.nq()], sizeof(double) * d.nq());
                if (d.maux > 0) std::memcpy(&naux[(size_t)i * d.naux()], &aux[(size_t)old * d.naux()], sizeof(double) * d.naux());
            } else {
                const fc2d_b200_options_t& oi = io[P.inst];
                if (d.maux > 0) app_setaux(oi, d, P, &naux[(size_t)i * d.naux()]);
                app_qinit(oi, d, P, d.maux > 0 ? &naux[(size_t)i * d.naux()] : nullptr, &nq[(size_t)i * d.nq()]);
            }
        }
        f = std::move(nf);
        q.swap(nq); aux.swap(naux);
    }
    std::vector<Leaf> L;
    for (const auto& P : f.p) L.push_back({P.level, P.gx, P.gy, P.inst});
    int rc = install_forest(s, L);
    if (rc) return rc;
    // install_forest sorted identically (same keys) -> same slot order as f
    CK(cudaMemcpyAsync(s->q, q.data(), q.size() * sizeof(double), cudaMemcpyHostToDevice, s->st));
    if (d.maux > 0) CK(cudaMemcpyAsync(s->aux, aux.data(), aux.size() * sizeof(double), cudaMemcpyHostToDevice, s->st));
    if (s->sphere) {
        // every patch's metric from scratch (fclaw2d_metric_patch_build), then its aux
        std::vector<MetricOp> ops(s->forest.np());
        for (int i = 0; i < s->forest.np(); i++) ops[i] = MetricOp{0, i, {0, 0, 0, 0}};
        CK(s->metric_dev.assign(ops, s->st));
        launch_sphere_metric(d, s->metric_dev.p, (int)ops.size(), 0, s->desc, s->o.maxlevel, nullptr, s->area, s->aux,
                             s->flow, s->st);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(s->st));
    s->t_curr = 0;
    s->initialized = true;
    return 0;
}

extern "C" int fc2d_b200_num_patches(const fc2d_b200_solver_t* s, int* np)
{
    if (!s || !np) return fail(FC2D_B200_EINVAL, "null argument");
    *np = s->forest.np();
    return 0;
}

extern "C" int fc2d_b200_patch_info(const fc2d_b200_solver_t* s, int* level, int* block, int* gx, int* gy)
{
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    for (int i = 0; i < s->forest.np(); i++) {
        const PatchInfo& P = s->forest.p[i];
        if (level) level[i] = P.level + s->forest.gi(P.inst).lbase;
        if (block) block[i] = P.block;
        if (gx) gx[i] = P.gx;
        if (gy) gy[i] = P.gy;
    }
    return 0;
}

extern "C" int fc2d_b200_get_q(fc2d_b200_solver_t* s, double* q)
{
    DeviceScope dev_scope_(s);
    if (!s || !q) return fail(FC2D_B200_EINVAL, "null argument");
    CK(cudaMemcpyAsync(q, s->q, (size_t)s->forest.np() * s->d.nq() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

extern "C" int fc2d_b200_set_q(fc2d_b200_solver_t* s, const double* q)
{
    DeviceScope dev_scope_(s);
    if (!s || !q) return fail(FC2D_B200_EINVAL, "null argument");
    CK(cudaMemcpyAsync(s->q, q, (size_t)s->forest.np() * s->d.nq() * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    std::memset(s->phys_ok, 0, sizeof(s->phys_ok));   // ghost cells are the caller's values
    return 0;
}

extern "C" int fc2d_b200_get_aux(fc2d_b200_solver_t* s, double* aux)
{
    DeviceScope dev_scope_(s);
    if (!s || !aux) return fail(FC2D_B200_EINVAL, "null argument");
    if (s->d.maux == 0) return 0;
    CK(cudaMemcpyAsync(aux, s->aux, (size_t)s->forest.np() * s->d.naux() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

extern "C" int fc2d_b200_set_aux(fc2d_b200_solver_t* s, const double* aux)
{
    DeviceScope dev_scope_(s);
    if (!s || !aux) return fail(FC2D_B200_EINVAL, "null argument");
    if (s->d.maux == 0) return 0;
    const size_t n = (size_t)s->forest.np() * s->d.naux();
    CK(cudaMemcpyAsync(s->aux, aux, n * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

extern "C" int fc2d_b200_registers_size(const fc2d_b200_solver_t* s, int* n)
{
    if (!s || !n) return fail(FC2D_B200_EINVAL, "null argument");
    *n = s->d.nreg();
    return 0;
}

extern "C" int fc2d_b200_get_registers(fc2d_b200_solver_t* s, double* r)
{
    DeviceScope dev_scope_(s);
    if (!s || !r) return fail(FC2D_B200_EINVAL, "null argument");
    CK(cudaMemcpyAsync(r, s->regs, (size_t)s->forest.np() * s->d.nreg() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

static int begin_cfl(fc2d_b200_solver* s)
{
    CK(cudaMemsetAsync(s->cfl_dev, 0, sizeof(unsigned long long) * s->ncfl, s->st));
    CK(cudaMemsetAsync(s->status_dev, 0, sizeof(unsigned int), s->st));
    return 0;
}

// The kernels' failure reports (device status word) as an error message, or "".
static std::string status_message(unsigned st)
{
    std::string m;
    if (st & STATUS_NONFINITE) m += "a non-finite value in q; ";
    if (st & STATUS_DEPTH) m += "negative water depth; ";
    if (st & STATUS_NEWTON) m += "the exact Riemann solver's Newton iteration on p* converged neither from its seed nor from PVRS; ";
    if (st & STATUS_STAGING) m += "a patch's copy into shared memory did not complete; ";
    if (!m.empty()) m.resize(m.size() - 2);
    return m;
}

// Level CFL maximum (over all instances); per instance into cfl_inst if given.
static int end_cfl(fc2d_b200_solver* s, double* cfl, double* cfl_inst = nullptr)
{
    CK(cudaMemcpyAsync(s->cfl_host, s->cfl_dev, sizeof(unsigned long long) * s->ncfl, cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(s->status_host, s->status_dev, sizeof(unsigned int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    unsigned status = *s->status_host;
    double v = 0.0;
    bool bad = false;
    for (int i = 0; i < s->ncfl; i++) {
        const double c = bits_to_double(s->cfl_host[i]);
        if (!(c == c)) bad = true;
        if (c > v) v = c;
        if (cfl_inst) cfl_inst[i] = c;
    }
    if (s->part) {
        // the CFL number and the failures of every rank (src/fclaw2d_run.c:206)
        double r[3] = {v, (double)status, bad ? 1.0 : 0.0};
        const bool xfail = s->part->failed;
        s->part->failed = false;
        if (s->part->comm.allreduce_max(s->part->comm.user, r, 3))
            return fail(FC2D_B200_ECUDA, "the allreduce callback failed");
        v = r[0]; status = (unsigned)r[1]; bad = r[2] != 0.0;
        if (xfail) return fail(FC2D_B200_ECUDA, "a halo exchange of this advance failed");
    }
    if (status) {
        if (cfl) *cfl = bits_to_double(0x7ff8000000000000ull);
        return fail(FC2D_B200_EDEVICE, "device status: " + status_message(status));
    }
    if (cfl) *cfl = bad ? bits_to_double(0x7ff8000000000000ull) : v;
    if (bad) return fail(FC2D_B200_EDEVICE, "non-finite CFL (negative depth or NaN in the update)");
    return 0;
}

extern "C" int fc2d_b200_level_update(fc2d_b200_solver_t* s, int level, double t, double dt, double* cfl)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    int rc = begin_cfl(s);
    if (rc) return rc;
    s->n_upd = 0;
    s->pend.active = false;
    s->emit = true; s->fill = true;
    rc = update_level(s, level, t, dt);
    if (rc) return rc;
    rc = flush_updates(s);
    if (rc) return rc;
    return end_cfl(s, cfl);
}

extern "C" int fc2d_b200_single_step_update(fc2d_b200_solver_t* s, int level, int iter, int total_count, double t,
                                            double dt, double* cfl)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    if (iter == 0) { s->ss_level = level; s->ss_count = 0; }
    if (level != s->ss_level || iter != s->ss_count) return fail(FC2D_B200_ESTATE, "single_step_update calls out of order");
    s->ss_count++;
    if (cfl) *cfl = 0.0;
    if (iter + 1 < total_count) return 0;
    const int np = s->forest.lev_off[level + 1] - s->forest.lev_off[level];
    if (total_count != np) return fail(FC2D_B200_ESTATE, "total_count differs from the patch count of the level");
    s->ss_level = -1;
    return fc2d_b200_level_update(s, level, t, dt, cfl);
}

// The buffering protocol with the patch data in the caller's host arrays.  The last
// call gathers the level's arrays into pinned staging in slot order, copies them to
// the level's (contiguous) device slots in one transfer, updates the level and
// scatters the result back the same way.
extern "C" int fc2d_b200_single_step_update_host(fc2d_b200_solver_t* s, int level, int gx, int gy, double* q,
                                                 const double* aux, int iter, int total_count, double t, double dt,
                                                 double* cfl)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    if (!q) return fail(FC2D_B200_EINVAL, "null patch array");
    if (!s->insts.empty() || s->part) return fail(FC2D_B200_EINVAL, "the host-data protocol drives one forest on one rank");
    if (iter == 0) { s->ss_level = level; s->ss_count = 0; s->ss_host.clear(); }
    if (level != s->ss_level || iter != s->ss_count) return fail(FC2D_B200_ESTATE, "single_step_update calls out of order");
    const Forest& f = s->forest;
    const int slot = f.lookup(0, level, gx, gy);
    if (slot < 0) return fail(FC2D_B200_EINVAL, "no patch of level " + std::to_string(level) + " at (" +
                                                     std::to_string(gx) + ", " + std::to_string(gy) + ")");
    s->ss_host.push_back({slot, q, aux});
    s->ss_count++;
    if (cfl) *cfl = 0.0;
    if (iter + 1 < total_count) return 0;
    s->ss_level = -1;
    const int p0 = f.lev_off[level], np = f.lev_off[level + 1] - p0;
    if (total_count != np || (int)s->ss_host.size() != np)
        return fail(FC2D_B200_ESTATE, "total_count differs from the patch count of the level");
    std::vector<char> seen(np, 0);
    for (const auto& h : s->ss_host) {
        if (seen[h.slot - p0]) return fail(FC2D_B200_EINVAL, "a patch was handed over twice");
        seen[h.slot - p0] = 1;
    }
    const size_t nq = s->d.nq(), na = s->d.naux();
    const size_t need = (size_t)np * (nq > na ? nq : na);
    if (s->ss_stage_cap < need) {
        if (s->ss_stage) CK(cudaFreeHost(s->ss_stage));
        s->ss_stage = nullptr;
        s->ss_stage_cap = 0;
        CK(cudaMallocHost(&s->ss_stage, need * sizeof(double)));
        s->ss_stage_cap = need;
    }
    CK(cudaStreamSynchronize(s->st));                  // the staging buffer is free
    if (na > 0 && s->ss_host[0].aux) {
        for (const auto& h : s->ss_host) {
            if (!h.aux) return fail(FC2D_B200_EINVAL, "aux given for some patches of the level only");
            std::memcpy(s->ss_stage + (size_t)(h.slot - p0) * na, h.aux, na * sizeof(double));
        }
        CK(cudaMemcpyAsync(s->aux + (size_t)p0 * na, s->ss_stage, (size_t)np * na * sizeof(double),
                           cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    for (const auto& h : s->ss_host) std::memcpy(s->ss_stage + (size_t)(h.slot - p0) * nq, h.q, nq * sizeof(double));
    CK(cudaMemcpyAsync(s->q + (size_t)p0 * nq, s->ss_stage, (size_t)np * nq * sizeof(double), cudaMemcpyHostToDevice,
                       s->st));
    int rc = fc2d_b200_level_update(s, level, t, dt, cfl);
    if (rc) return rc;
    CK(cudaMemcpyAsync(s->ss_stage, s->q + (size_t)p0 * nq, (size_t)np * nq * sizeof(double), cudaMemcpyDeviceToHost,
                       s->st));
    CK(cudaStreamSynchronize(s->st));
    for (const auto& h : s->ss_host) std::memcpy(h.q, s->ss_stage + (size_t)(h.slot - p0) * nq, nq * sizeof(double));
    s->ss_host.clear();
    return 0;
}

extern "C" int fc2d_b200_ghost_update(fc2d_b200_solver_t* s, int minlevel, int maxlevel, double sync_time, int time_interp)
{
    DeviceScope dev_scope_(s);
    (void)sync_time;
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    if (time_interp && !s->qinterp) return fail(FC2D_B200_EINVAL, "time interpolation needs subcycle");
    ghost_update(s, minlevel, maxlevel, time_interp);
    (void)flush_pending(s);
    CK(cudaGetLastError());
    return 0;
}

extern "C" int fc2d_b200_timeinterp(fc2d_b200_solver_t* s, int level, double alpha)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized || !s->qinterp) return fail(FC2D_B200_ESTATE, "time interpolation needs subcycle");
    timeinterp(s, level, alpha);
    (void)flush_pending(s);
    CK(cudaGetLastError());
    return 0;
}

extern "C" int fc2d_b200_time_sync(fc2d_b200_solver_t* s, int minlevel, int maxlevel)
{
    DeviceScope dev_scope_(s);
    if (s && s->part && s->initialized) {
        int rc = halo_exchange(s, false);          // the registers of other ranks' patches
        if (rc) return rc;
    }
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    time_sync(s, minlevel, maxlevel);
    (void)flush_pending(s);
    CK(cudaGetLastError());
    return 0;
}

// One pass of fclaw2d_advance_all_levels over the current forest.
static int traverse_advance(fc2d_b200_solver* s, double t, double dt)
{
    const fc2d_b200_options_t& o = s->o;
    Tsc ts[34];
    std::memset(ts, 0, sizeof(ts));
    const int minlevel = s->forest.minlevel_present, maxlevel = s->forest.maxlevel_present;
    for (int l = o.minlevel; l <= o.maxlevel; l++) { ts[l].last_step = 0; ts[l].current_time = t; }
    if (o.subcycle) {
        double dt_level = dt;
        int steps_inc = 1 << (maxlevel - o.minlevel);
        int total = 1;
        for (int l = o.minlevel; l <= o.maxlevel; l++) {
            ts[l].dt_step = dt_level; ts[l].total_steps = total; ts[l].step_inc = steps_inc;
            dt_level /= 2; steps_inc /= 2; total *= 2;
        }
    } else {
        const int rf = 1 << (o.maxlevel - o.minlevel);
        for (int l = o.minlevel; l <= o.maxlevel; l++) { ts[l].step_inc = 1; ts[l].dt_step = dt / rf; ts[l].total_steps = rf; }
    }
    s->n_upd = 0;
    s->pend.active = false;
    s->pend_ti.active = false;
    const int nfine = ts[maxlevel].total_steps;
    for (int nf = 0; nf < nfine; nf++) {
        int rc = advance_level(s, ts, maxlevel, nf);
        if (rc) return rc;
        if (ts[maxlevel].last_step < ts[maxlevel].total_steps) {
            if (o.subcycle) {
                int ti = maxlevel - 1;
                while (ts[maxlevel].last_step % ts[ti].step_inc == 0) ti--;
                ghost_update(s, ti + 1, maxlevel, 1);
                if (o.time_sync) time_sync(s, ti + 1, maxlevel, true);
            } else {
                ghost_update(s, minlevel, maxlevel, 0);
                if (o.time_sync) time_sync(s, minlevel, maxlevel, true);
            }
        }
    }
    ghost_update(s, minlevel, maxlevel, 0);
    if (o.time_sync) time_sync(s, minlevel, maxlevel);
    return flush_pending(s);
}

// First half of an advance: host traversal, parameter upload and the launches
// (graph replay); returns without waiting for the device.
static int advance_launch(fc2d_b200_solver_t* s, double t, double dt)
{
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    const double h0 = wall_ms();
    s->ev_used = 0;
    s->upd_launch_bytes.clear();
    s->upd_launches = 0;
    s->total_launches = 0;
    // pass 1: host traversal filling the per-launch parameters and statistics
    s->emit = false; s->fill = true;
    int rc = traverse_advance(s, t, dt);
    if (rc) { s->emit = true; return rc; }
    s->step_host_ms = wall_ms() - h0;
    if (!s->step_ev[0]) {
        CK(cudaEventCreate(&s->step_ev[0]));
        CK(cudaEventCreate(&s->step_ev[1]));
    }
    CK(cudaEventRecord(s->step_ev[0], s->st));
    ProgrammaticScope pscope(s->programmatic);
    const int nupd = s->n_upd;
    rc = begin_cfl(s);
    if (rc) return rc;
    if (nupd) CK(cudaMemcpyAsync(s->params_dev, s->params_host, sizeof(StepParams) * nupd, cudaMemcpyHostToDevice, s->st));
    // pass 2: the launches, captured once per forest into a CUDA graph and replayed
    s->emit = true; s->fill = false;
    if (s->use_graphs && !s->timing) {
        if (s->graph_stale || !s->graph_exec || s->graph_nupd != nupd) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
            rc = traverse_advance(s, t, dt);
            cudaError_t ec = cudaStreamEndCapture(s->st, &g);
            if (rc) { if (g) cudaGraphDestroy(g); s->fill = true; return rc; }
            if (ec != cudaSuccess) { s->fill = true; return fail(FC2D_B200_ECUDA, std::string("graph capture: ") + cudaGetErrorString(ec)); }
            bool updated = false;
            if (s->graph_exec) {
                // same launches with new grids and arguments (a regrid): new parameters in place
                cudaGraphExecUpdateResultInfo info{};
                updated = cudaGraphExecUpdate(s->graph_exec, g, &info) == cudaSuccess;
                if (!updated) { (void)cudaGetLastError(); release_graph(s); }
            }
            if (!updated) {
                ec = cudaGraphInstantiate(&s->graph_exec, g, 0);
                if (ec != cudaSuccess) {
                    cudaGraphDestroy(g);
                    s->graph_exec = nullptr; s->fill = true;
                    return fail(FC2D_B200_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ec));
                }
                s->graph_builds++;
            } else {
                s->graph_updates++;
            }
            cudaGraphDestroy(g);
            s->graph_stale = false;
            s->graph_nupd = nupd;
        }
        CK(cudaGraphLaunch(s->graph_exec, s->st));
    } else {
        rc = traverse_advance(s, t, dt);
    }
    s->fill = true;
    if (rc) return rc;
    CK(cudaGetLastError());
    CK(cudaEventRecord(s->step_ev[1], s->st));
    s->pending_t = t + dt;
    s->pending = true;
    return 0;
}

// Second half: wait for the solver's stream, CFL maximum (per instance into
// cfl_inst), timing statistics.
static int advance_finish(fc2d_b200_solver_t* s, double* maxcfl, double* cfl_inst)
{
    if (!s->pending) return fail(FC2D_B200_ESTATE, "no advance in flight");
    s->pending = false;
    int rc = end_cfl(s, maxcfl, cfl_inst);
    {
        float m = 0;
        if (s->step_ev[0] && cudaEventElapsedTime(&m, s->step_ev[0], s->step_ev[1]) == cudaSuccess) s->step_device_ms = m;
        else { (void)cudaGetLastError(); s->step_device_ms = 0; }
    }
    if (s->timing) {
        double ms = 0, bytes = 0;
        for (auto& pr : s->upd_launch_bytes) {
            float m = 0;
            CK(cudaEventElapsedTime(&m, s->ev_pool[pr.first], s->ev_pool[pr.first + 1]));
            ms += m;
            bytes += pr.second;
        }
        s->upd_ms = ms;
        s->upd_bytes = bytes;
    }
    s->t_curr = s->pending_t;
    return rc;
}

extern "C" int fc2d_b200_advance(fc2d_b200_solver_t* s, double t, double dt, double* maxcfl)
{
    DeviceScope dev_scope_(s);
    if (s && s->pending) return fail(FC2D_B200_ESTATE, "an advance is in flight");
    int rc = advance_launch(s, t, dt);
    if (rc) return rc;
    return advance_finish(s, maxcfl, nullptr);
}

extern "C" int fc2d_b200_regrid(fc2d_b200_solver_t* s, int* changed_out)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    const double t_start = wall_ms();
    for (double& v : s->regrid_ms) v = 0.0;
    const Dims& d = s->d;
    const Forest& f = s->forest;
    const int np = f.np();
    std::vector<int> flags(np);
    CK(s->flags_dev.assign(flags, s->st));
    const int crit = tag_criterion(s->o);
    const bool minmax = crit == FC2D_B200_TAG_MINMAX;
    const int mq = s->o.threshold_variable > 0 ? s->o.threshold_variable - 1 : 0;
    std::vector<double> mm;
    if (minmax) {
        mm.assign(2 * (size_t)np, 0.0);
        CK(s->minmax_dev.assign(mm, s->st));
    }
    launch_tag(d, s->q, s->desc, np, crit, mq, s->o.refine_threshold, s->o.coarsen_threshold, s->flags_dev.p, s->st,
               minmax ? s->minmax_dev.p : nullptr);
    CK(cudaMemcpyAsync(flags.data(), s->flags_dev.p, sizeof(int) * (size_t)np, cudaMemcpyDeviceToHost, s->st));
    if (minmax) CK(cudaMemcpyAsync(mm.data(), s->minmax_dev.p, sizeof(double) * mm.size(), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (s->part) {
        // each rank's tags are valid for its own patches only: reduce them over ranks
        // (other ranks' entries as -1, ranges as +inf / -inf)
        auto& P = *s->part;
        std::vector<double> r((size_t)np * (minmax ? 3 : 1));
        for (int i = 0; i < np; i++) {
            const bool me = P.plan.owner[i] == P.comm.rank;
            r[i] = me ? (double)flags[i] : -1.0;
            if (minmax) {
                r[np + i] = me ? -mm[2 * i] : -INFINITY;
                r[2 * (size_t)np + i] = me ? mm[2 * i + 1] : -INFINITY;
            }
        }
        if (P.comm.allreduce_max(P.comm.user, r.data(), (int)r.size()))
            return fail(FC2D_B200_ECUDA, "the allreduce callback failed");
        for (int i = 0; i < np; i++) {
            flags[i] = (int)r[i];
            if (minmax) { mm[2 * i] = -r[np + i]; mm[2 * i + 1] = r[2 * (size_t)np + i]; }
        }
    }
    const double t_mark = wall_ms();
    s->regrid_ms[0] = t_mark - t_start;
    // clawpatch_tag4refinement / _tag4coarsening (fclaw2d_clawpatch.cpp:800-910): a negative
    // refine threshold always refines, a threshold <= 0 never coarsens
    const bool always_refine = s->o.refine_threshold < 0, never_coarsen = !(s->o.coarsen_threshold > 0);
    // cb_regrid_tag4coarsening (families) then cb_fclaw2d_regrid_tag4refinement
    std::vector<int> mark(np, 0);
    for (int i = 0; i < np; i++) {
        const PatchInfo& P = f.p[i];
        if (P.level <= inst_minlev(s, P.inst) || (P.gx & 1) || (P.gy & 1)) continue;
        int sib[4]; bool ok = true;
        for (int k = 0; k < 4; k++) {
            sib[k] = f.lookup(P.inst, P.level, P.gx + (k & 1), P.gy + (k >> 1));
            if (sib[k] < 0) { ok = false; break; }
        }
        if (!ok) continue;
        bool coarsen = !never_coarsen;
        if (never_coarsen) {
        } else if (minmax) {
            // minmax over the family (fclaw2d_clawpatch46_fort_tag4coarsening.f:35-58)
            double lo = mm[2 * sib[0]], hi = mm[2 * sib[0] + 1];
            for (int k = 1; k < 4; k++) { lo = std::min(lo, mm[2 * sib[k]]); hi = std::max(hi, mm[2 * sib[k] + 1]); }
            coarsen = !(hi - lo > s->o.coarsen_threshold);
        } else {
            for (int k = 0; k < 4; k++) if (!(flags[sib[k]] & 2)) coarsen = false;
        }
        if (coarsen) for (int k = 0; k < 4; k++) mark[sib[k]] = -1;
    }
    for (int i = 0; i < np; i++)
        if (f.p[i].level < inst_maxlev(s, f.p[i].inst) && (always_refine || (flags[i] & 1))) mark[i] = 1;
    if (s->o.smooth_refine) smooth_marks(f, mark, s->o.smooth_level);
    int changed = 0;
    std::string err;
    std::vector<Leaf> L = adapt_leaves(f, mark, changed, err);
    if (changed_out) *changed_out = changed;
    const double t_adapt = wall_ms();
    s->regrid_ms[1] = t_adapt - t_mark;
    if (!changed) { s->regrid_ms[7] = t_adapt - t_start; return 0; }
    if (s->part) {
        // repopulation reads old patches any rank may own: every rank gets all of them
        int rc = halo_exchange(s, true);
        if (rc) return rc;
    }
    Forest& nf = s->forest_next;                 // built in place: its buffers stay from the last regrid
    nf.g = f.g;
    nf.inst = f.inst;
    if (!nf.build(L, err)) return fail(FC2D_B200_EFOREST, err);
    const double t_build = wall_ms();
    s->regrid_ms[2] = t_build - t_adapt;
    // batch: an instance without an applied refinement or family coarsening
    // keeps its ghost cells, as it would alone (fclaw2d_regrid does no ghost
    // update then); a coarsening that balance refines again still counts as a change
    std::vector<int> keep;
    if (!s->insts.empty()) {
        std::vector<int> adapted(nf.ninst(), 0);
        for (int i = 0; i < np; i++) {
            const PatchInfo& P = f.p[i];
            if (mark[i] > 0) adapted[P.inst] = 1;
            if (mark[i] < 0) {
                bool all = true;
                for (int k = 0; k < 4; k++) {
                    const int j = f.lookup(P.inst, P.level, 2 * (P.gx >> 1) + (k & 1), 2 * (P.gy >> 1) + (k >> 1));
                    if (j < 0 || mark[j] >= 0) all = false;
                }
                if (all) adapted[P.inst] = 1;
            }
        }
        for (int i = 0; i < nf.np(); i++)
            if (!adapted[nf.p[i].inst]) keep.push_back(i);
    }
    // repopulation ops (cb_fclaw2d_regrid_repopulate)
    std::vector<RepopOp> ops(nf.np());
    // aux of the new forest, filled on the device: a kept patch's from the old slab
    // (asrc = old slot), a new patch's from the app's setaux on the host (staged,
    // asrc = -2 - k) or from the cubed-sphere metric (asrc = -1)
    std::vector<int> asrc(d.maux > 0 ? nf.np() : 0);
    std::vector<double> staged;
    for (int i = 0; i < nf.np(); i++) {
        const PatchInfo& P = nf.p[i];
        RepopOp op{};
        op.dst = i;
        const int old = f.lookup(P.inst, P.level, P.gx, P.gy);
        if (old >= 0) {
            op.kind = 0; op.src = old;
            if (d.maux > 0) asrc[i] = old;
        } else {
            const int parent = f.lookup(P.inst, P.level - 1, P.gx >> 1, P.gy >> 1);
            if (parent >= 0) { op.kind = 1; op.src = parent; op.igrid = (P.gx & 1) + 2 * (P.gy & 1); }
            else {
                op.kind = 2;
                for (int c = 0; c < 4; c++) {
                    op.child[c] = f.lookup(P.inst, P.level + 1, 2 * P.gx + (c & 1), 2 * P.gy + (c >> 1));
                    if (op.child[c] < 0) return fail(FC2D_B200_EFOREST, "adapt jumped more than one level");
                }
            }
            if (d.maux > 0 && s->sphere) asrc[i] = -1;
            else if (d.maux > 0) {
                const size_t k = staged.size() / d.naux();
                staged.resize(staged.size() + d.naux(), 0.0);
                app_setaux(inst_options(s, P.inst), d, P, &staged[k * d.naux()]);
                asrc[i] = -2 - (int)k;
            }
        }
        ops[i] = op;
    }
    // repopulate into the spare slabs, then swap them with the current ones
    int rc = ensure_spare(s, nf.np());
    if (rc) return rc;
    auto& sp = s->spare;
    CK(s->repop_dev.assign(ops, s->st));
    if (d.maux > 0) {
        CK(s->aux_src_dev.assign(asrc, s->st));
        if (!staged.empty()) CK(s->aux_staged_dev.assign(staged, s->st));
        launch_aux_repop(d, s->aux_src_dev.p, nf.np(), s->aux, s->aux_staged_dev.p, sp.aux, s->st);
    }
    std::vector<PatchDesc> hd;
    if (s->sphere) {
        // metric of the new forest before repopulation, which weights by the areas:
        // kept patches copy, refined ones build from scratch, coarsened ones from their
        // children (cb_fclaw2d_regrid_repopulate: fclaw2d_patch_build / _build_from_fine)
        // (new patches first, then the kept ones)
        std::vector<MetricOp> mops, kept;
        for (size_t i = 0; i < ops.size(); i++) {
            const RepopOp& o = ops[i];
            if (o.kind == 0) kept.push_back(MetricOp{1, (int)i, {o.src, 0, 0, 0}});
            else if (o.kind == 1) mops.push_back(MetricOp{0, (int)i, {0, 0, 0, 0}});
            else mops.push_back(MetricOp{2, (int)i, {o.child[0], o.child[1], o.child[2], o.child[3]}});
        }
        const int nnew = (int)mops.size(), nkept = (int)kept.size();
        mops.insert(mops.end(), kept.begin(), kept.end());
        hd = make_desc(nf);
        CK(cudaMemcpyAsync(sp.desc, hd.data(), hd.size() * sizeof(PatchDesc), cudaMemcpyHostToDevice, s->st));
        CK(s->metric_dev.assign(mops, s->st));
        launch_sphere_metric(d, s->metric_dev.p, nnew, nkept, sp.desc, s->o.maxlevel, s->area, sp.area, sp.aux,
                             s->flow, s->st);
    }
    launch_repop(d, s->repop_dev.p, (int)ops.size(), s->q, sp.q, s->qlast, sp.qlast, s->qinterp, sp.qinterp, s->regs,
                 sp.regs, s->sphere ? s->area : nullptr, s->sphere ? sp.area : nullptr, s->st);
    CK(cudaGetLastError());       // the repopulation runs while the host builds the tables below
    std::swap(s->q, sp.q); std::swap(s->qlast, sp.qlast); std::swap(s->qinterp, sp.qinterp);
    std::swap(s->aux, sp.aux); std::swap(s->regs, sp.regs); std::swap(s->desc, sp.desc);
    std::swap(s->area, sp.area);
    std::swap(s->cap, sp.cap);
    std::swap(s->forest, s->forest_next);
    s->forest_gen++;
    invalidate_graph(s);
    const double t_repop = wall_ms();
    s->regrid_ms[3] = t_repop - t_build;
    rc = upload_desc_and_tables(s);
    if (rc) return rc;
    const double t_upload = wall_ms();
    s->regrid_ms[5] = t_upload - t_repop - s->regrid_ms[4];
    if (!keep.empty()) {
        const size_t nq_all = (size_t)s->forest.np() * d.nq();
        if (s->snap.cap < nq_all) {
            std::vector<double> sz(nq_all);
            CK(s->snap.assign(sz, s->st));
        }
        CK(cudaMemcpyAsync(s->snap.p, s->q, sizeof(double) * nq_all, cudaMemcpyDeviceToDevice, s->st));
        CK(s->keep_dev.assign(keep, s->st));
    }
    unsigned char phys_before[64];
    std::memcpy(phys_before, s->phys_ok, sizeof(phys_before));
    ghost_update(s, s->forest.minlevel_present, s->forest.maxlevel_present, 0);
    if (!keep.empty()) {
        launch_restore_patches(d, s->q, s->snap.p, s->keep_dev.p, (int)keep.size(), s->st);
        // kept instances have their old ghost cells back
        for (int k : keep) {
            const int l = s->forest.p[k].level;
            if (l >= 0 && l < 64) s->phys_ok[l] = s->phys_ok[l] && phys_before[l];
        }
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->st));
    const double t_end = wall_ms();
    s->regrid_ms[6] = t_end - t_upload;
    s->regrid_ms[7] = t_end - t_start;
    return 0;
}

extern "C" int fc2d_b200_last_regrid_stats(const fc2d_b200_solver_t* s, double* ms)
{
    if (!s || !ms) return fail(FC2D_B200_EINVAL, "null argument");
    for (int k = 0; k < 8; k++) ms[k] = s->regrid_ms[k];
    return 0;
}

// ---------------------------------------------------------------------------
// save / restore a step and the run loop (src/fclaw2d_run.c)
// ---------------------------------------------------------------------------
extern "C" int fc2d_b200_save_step(fc2d_b200_solver_t* s)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    if (s->pending) return fail(FC2D_B200_ESTATE, "an advance is in flight");
    CK(cudaSetDevice(s->o.device));
    const size_t n = (size_t)s->forest.np() * s->d.nq();
    if (s->qsave_cap < n) {
        if (s->qsave) CK(cudaFree(s->qsave));
        s->qsave = nullptr;
        s->qsave_cap = 0;
        CK(cudaMalloc(&s->qsave, n * sizeof(double)));
        s->qsave_cap = n;
    }
    CK(cudaMemcpyAsync(s->qsave, s->q, n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    s->qsave_n = n;
    s->qsave_gen = s->forest_gen;
    std::memcpy(s->phys_ok_save, s->phys_ok, sizeof(s->phys_ok));
    return 0;
}

extern "C" int fc2d_b200_restore_step(fc2d_b200_solver_t* s)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    if (s->pending) return fail(FC2D_B200_ESTATE, "an advance is in flight");
    const size_t n = (size_t)s->forest.np() * s->d.nq();
    if (s->qsave_n != n || s->qsave_gen != s->forest_gen)
        return fail(FC2D_B200_ESTATE, "no saved step for the current forest");
    CK(cudaSetDevice(s->o.device));
    CK(cudaMemcpyAsync(s->q, s->qsave, n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    // the ghost cells are back to their saved values, physical ones included
    std::memcpy(s->phys_ok, s->phys_ok_save, sizeof(s->phys_ok));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

// outstyle_1 (src/fclaw2d_run.c:113-265) with reduce_cfl (one process: the global
// maximum is the local one) and advance_one_step off.
extern "C" int fc2d_b200_run(fc2d_b200_solver_t* s, fc2d_b200_run_stats_t* out)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    if (!s->insts.empty()) return fail(FC2D_B200_EINVAL, "fc2d_b200_run drives one forest; batches step by advance_instances");
    const fc2d_b200_options_t& o = s->o;
    if (!(o.tfinal > 0) || !(o.initial_dt > 0)) return fail(FC2D_B200_EINVAL, "fc2d_b200_run needs tfinal > 0 and initial_dt > 0");
    fc2d_b200_run_stats_t st{};
    const int nout = o.nout > 0 ? o.nout : 1;
    double dt_minlevel = o.initial_dt;
    const double t0 = 0;
    const double dt_outer = (o.tfinal - t0) / ((double)nout);
    double t_curr = t0;
    int n_inner = 0, retakes = 0;
    for (int n = 0; n < nout; n++) {
        const double tstart = t_curr;
        const double tend = tstart + dt_outer;
        while (t_curr < tend) {
            int rc;
            if (!o.use_fixed_dt && (rc = fc2d_b200_save_step(s))) return rc;
            // take a slightly larger step now rather than a tiny one to hit tend later
            double dt_step = dt_minlevel;
            const double tol = 1e-2 * dt_step;
            int took_small_step = 0;
            if (!o.use_fixed_dt) {
                const double small_step = tend - (t_curr + dt_step);
                if (small_step < tol) {
                    dt_step = tend - t_curr;
                    if (small_step < 0) took_small_step = 1;
                }
            }
            if (!(dt_step > 0) || !std::isfinite(dt_step))
                return fail(FC2D_B200_EDEVICE, "fc2d_b200_run: the time step is " + std::to_string(dt_step) +
                                                   " at t = " + std::to_string(t_curr));
            double maxcfl_step = 0;
            if ((rc = fc2d_b200_advance(s, t_curr, dt_step, &maxcfl_step))) return rc;
            st.count_amr_advance++;
            if (!std::isfinite(maxcfl_step))
                return fail(FC2D_B200_EDEVICE, "fc2d_b200_run: non-finite CFL number (negative depth or NaN in q) at t = " +
                                                   std::to_string(t_curr));
            if (maxcfl_step > o.max_cfl && !o.use_fixed_dt) {
                // retake the step from the saved copy with a smaller dt
                if ((rc = fc2d_b200_restore_step(s))) return rc;
                if (++retakes > 64) return fail(FC2D_B200_EDEVICE, "fc2d_b200_run: 64 retakes of one step");
                dt_minlevel = dt_minlevel * o.desired_cfl / maxcfl_step;
                st.rejected++;
                continue;
            }
            retakes = 0;
            n_inner++;
            t_curr += dt_step;
            if (!o.use_fixed_dt) {
                const double dt_new = dt_minlevel * o.desired_cfl / maxcfl_step;
                if (!took_small_step) dt_minlevel = dt_new;
            }
            if (o.regrid_interval > 0 && n_inner % o.regrid_interval == 0) {
                int changed = 0;
                if ((rc = fc2d_b200_regrid(s, &changed))) return rc;
                st.count_amr_regrid++;
                if (changed) st.count_amr_new_domain++;
            }
        }
    }
    st.steps = n_inner;
    st.global_num_patches = s->forest.np();
    st.t_final = t_curr;
    if (out) *out = st;
    return 0;
}

// ---------------------------------------------------------------------------
// one forest over several ranks
// ---------------------------------------------------------------------------
extern "C" int fc2d_b200_set_partition(fc2d_b200_solver_t* s, const fc2d_b200_comm_t* comm)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    if (s->pending) return fail(FC2D_B200_ESTATE, "an advance is in flight");
    if (!comm) {
        if (s->part) {
            if (s->initialized) {                     // every rank gets the whole forest back
                int rc = halo_exchange(s, true);
                if (rc) return rc;
            }
            const bool g = s->part->graphs_before;
            if (s->part->buf) cudaFree(s->part->buf);
            s->part.reset();
            s->use_graphs = g;
            invalidate_graph(s);
            if (s->initialized) return upload_desc_and_tables(s);
        }
        return 0;
    }
    if (comm->size < 1 || comm->rank < 0 || comm->rank >= comm->size || !comm->exchange || !comm->allreduce_max ||
        !comm->allreduce_sum)
        return fail(FC2D_B200_EINVAL, "bad communicator (rank, size or a callback missing)");
    if (!s->insts.empty()) return fail(FC2D_B200_EINVAL, "batches of instances are distributed by instance, not partitioned");
    const bool g = s->part ? s->part->graphs_before : s->use_graphs;
    if (!s->part) s->part = std::make_unique<fc2d_b200_solver::PartState>();
    s->part->comm = *comm;
    s->part->graphs_before = g;
    s->use_graphs = false;                            // transfers run between the launches of an advance
    invalidate_graph(s);
    if (s->initialized) return upload_desc_and_tables(s);
    return 0;
}

extern "C" int fc2d_b200_partition_owner(const fc2d_b200_solver_t* s, int* owner)
{
    if (!s || !owner) return fail(FC2D_B200_EINVAL, "null argument");
    const int np = s->forest.np();
    for (int i = 0; i < np; i++) owner[i] = s->part ? s->part->plan.owner[i] : 0;
    return 0;
}

extern "C" int fc2d_b200_sync_replicas(fc2d_b200_solver_t* s)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized) return fail(FC2D_B200_ESTATE, "solver not initialized");
    if (s->pending) return fail(FC2D_B200_ESTATE, "an advance is in flight");
    if (!s->part) return 0;
    return halo_exchange(s, true);
}

extern "C" int fc2d_b200_partition_plan(const fc2d_b200_options_t* opt, int np, const int* level, const int* gx,
                                        const int* gy, int rank, int size, int* owner, int* nsend, int* nrecv,
                                        unsigned long long* send_sum, unsigned long long* recv_sum)
{
    if (!opt || np <= 0 || !level || !gx || !gy || !owner || size < 1 || rank < 0 || rank >= size)
        return fail(FC2D_B200_EINVAL, "bad arguments");
    const fc2d_b200_options_t& o = *opt;
    Forest f;
    const Dims d{o.mx, o.my, o.mbc, o.meqn, o.maux};
    f.g = Geometry{d, o.mi > 0 ? o.mi : 1, o.mj > 0 ? o.mj : 1, o.ax, o.bx, o.ay, o.by};
    if (o.app == FC2D_B200_APP_SPHERE) { f.g = Geometry{d, 6, 1, 0.0, 1.0, 0.0, 1.0}; f.g.kind = 1; }
    std::vector<Leaf> L(np);
    for (int i = 0; i < np; i++) L[i] = Leaf{level[i], gx[i], gy[i], 0};
    std::string err;
    if (!f.build(L, err)) return fail(FC2D_B200_EFOREST, err);
    PartitionPlan pl;
    make_partition(f, rank, size, pl);
    for (int i = 0; i < np; i++) owner[i] = pl.owner[i];
    for (int r = 0; r < size; r++) {
        if (nsend) nsend[r] = 0;
        if (nrecv) nrecv[r] = 0;
        if (send_sum) send_sum[r] = 0;
        if (recv_sum) recv_sum[r] = 0;
    }
    for (size_t k = 0; k < pl.peers.size(); k++) {
        const int r = pl.peers[k];
        if (nsend) nsend[r] = (int)pl.send[k].size();
        if (nrecv) nrecv[r] = (int)pl.recv[k].size();
        for (int v : pl.send[k]) if (send_sum) send_sum[r] += (unsigned long long)v * 2654435761ull + 1ull;
        for (int v : pl.recv[k]) if (recv_sum) recv_sum[r] += (unsigned long long)v * 2654435761ull + 1ull;
    }
    return 0;
}

extern "C" int fc2d_b200_mass(fc2d_b200_solver_t* s, double* out)
{
    DeviceScope dev_scope_(s);
    if (!s || !out || !s->initialized) return fail(FC2D_B200_EINVAL, "bad arguments");
    const int np = s->forest.np(), meqn = s->d.meqn;
    if (np * meqn > s->mass_cap) {
        if (s->mass_dev) cudaFree(s->mass_dev);
        s->mass_cap = np * meqn + 1024;
        CK(cudaMalloc(&s->mass_dev, sizeof(double) * (size_t)s->mass_cap));
    }
    launch_patch_mass(s->d, s->q, s->desc, np, s->mass_dev, s->st, s->area);
    std::vector<double> pm((size_t)np * meqn);
    CK(cudaMemcpyAsync(pm.data(), s->mass_dev, sizeof(double) * pm.size(), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (s->part) {
        // each patch's partial from its owner (the others add exact zeros), then the
        // Kahan sum over patches in order, as on one rank
        auto& P = *s->part;
        for (int p = 0; p < np; p++)
            if (P.plan.owner[p] != P.comm.rank)
                for (int m = 0; m < meqn; m++) pm[(size_t)p * meqn + m] = 0.0;
        if (P.comm.allreduce_sum(P.comm.user, pm.data(), (int)pm.size()))
            return fail(FC2D_B200_ECUDA, "the allreduce callback failed");
    }
    for (int m = 0; m < meqn; m++) {
        double sum = 0.0, comp = 0.0;
        for (int p = 0; p < np; p++) {
            const double y = pm[(size_t)p * meqn + m] - comp;
            const double t = sum + y;
            comp = (t - sum) - y;
            sum = t;
        }
        out[m] = sum;
    }
    return 0;
}

extern "C" int fc2d_b200_cell_updates(const fc2d_b200_solver_t* s, double* out)
{
    if (!s || !out) return fail(FC2D_B200_EINVAL, "null argument");
    *out = s->cell_updates;
    return 0;
}

extern "C" int fc2d_b200_synchronize(fc2d_b200_solver_t* s)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

extern "C" int fc2d_b200_last_update_stats(const fc2d_b200_solver_t* s, double* update_ms, double* update_bytes,
                                           int* update_launches, int* total_launches)
{
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    if (update_ms) *update_ms = s->upd_ms;
    if (update_bytes) *update_bytes = s->upd_bytes;
    if (update_launches) *update_launches = s->upd_launches;
    if (total_launches) *total_launches = s->total_launches;
    return 0;
}

extern "C" int fc2d_b200_graph_stats(const fc2d_b200_solver_t* s, int* builds, int* updates)
{
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    if (builds) *builds = s->graph_builds;
    if (updates) *updates = s->graph_updates;
    return 0;
}

extern "C" int fc2d_b200_last_step_timing(const fc2d_b200_solver_t* s, double* host_ms, double* device_ms)
{
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    if (host_ms) *host_ms = s->step_host_ms;
    if (device_ms) *device_ms = s->step_device_ms;
    return 0;
}

extern "C" int fc2d_b200_set_timing(fc2d_b200_solver_t* s, int enable)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    s->timing = enable != 0;
    return 0;
}

extern "C" int fc2d_b200_event_record(fc2d_b200_solver_t* s, int slot)
{
    DeviceScope dev_scope_(s);
    if (!s || slot < 0 || slot >= 64) return fail(FC2D_B200_EINVAL, "bad event slot");
    if (s->user_ev.empty()) {
        s->user_ev.resize(64);
        for (auto& e : s->user_ev) CK(cudaEventCreate(&e));
    }
    CK(cudaEventRecord(s->user_ev[slot], s->st));
    return 0;
}

extern "C" int fc2d_b200_event_elapsed(fc2d_b200_solver_t* s, int a, int b, double* ms)
{
    DeviceScope dev_scope_(s);
    if (!s || !ms || a < 0 || b < 0 || a >= (int)s->user_ev.size() || b >= (int)s->user_ev.size())
        return fail(FC2D_B200_EINVAL, "bad event slots");
    CK(cudaEventSynchronize(s->user_ev[b]));
    float m = 0;
    CK(cudaEventElapsedTime(&m, s->user_ev[a], s->user_ev[b]));
    *ms = m;
    return 0;
}

extern "C" int fc2d_b200_get_stream(const fc2d_b200_solver_t* s, void** stream)
{
    if (!s || !stream) return fail(FC2D_B200_EINVAL, "null argument");
    *stream = (void*)s->st;
    return 0;
}

extern "C" int fc2d_b200_set_programmatic_launch(fc2d_b200_solver_t* s, int enable)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    s->programmatic = enable != 0;
    invalidate_graph(s);
    return 0;
}

extern "C" int fc2d_b200_set_graphs(fc2d_b200_solver_t* s, int enable)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    if (s->part) { s->part->graphs_before = enable != 0; return 0; }   // eager while partitioned
    s->use_graphs = enable != 0;
    invalidate_graph(s);
    return 0;
}

extern "C" int fc2d_b200_mass_noalloc(fc2d_b200_solver_t* s, double* out)
{
    DeviceScope dev_scope_(s);
    if (!s || !out || !s->initialized) return fail(FC2D_B200_EINVAL, "bad arguments");
    if (s->part) return fail(FC2D_B200_EINVAL, "fc2d_b200_mass_noalloc covers one rank; a partitioned forest uses fc2d_b200_mass");
    if (s->sphere) return fail(FC2D_B200_EINVAL, "fc2d_b200_mass_noalloc weights by dx dy; a manifold needs fc2d_b200_mass");
    const long long np = s->forest.np(), meqn = s->d.meqn;
    if (np * meqn + meqn > (long long)MASS_SCRATCH_DOUBLES)
        return fail(FC2D_B200_EINVAL, "fc2d_b200_mass_noalloc: npatches*meqn + meqn = " + std::to_string(np * meqn + meqn) +
                                          " exceeds the static scratch of " + std::to_string((int)MASS_SCRATCH_DOUBLES) +
                                          " doubles; use fc2d_b200_mass");
    double* scratch = nullptr;
    int rc = scratch_for_device(s->o.device, &scratch);
    if (rc) return rc;
    launch_mass_noalloc(s->d, s->q, s->desc, (int)np, scratch, s->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, scratch + np * meqn, sizeof(double) * (size_t)meqn, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

extern "C" int fc2d_b200_newton_histogram(fc2d_b200_solver_t* s, unsigned long long* out, int reset)
{
    DeviceScope dev_scope_(s);
    if (!s || !out) return fail(FC2D_B200_EINVAL, "null argument");
    CK(cudaMemcpyAsync(out, s->newton_hist, 32 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (reset) {
        CK(cudaMemsetAsync(s->newton_hist, 0, 32 * sizeof(unsigned long long), s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    return 0;
}

// ---------------------------------------------------------------------------
// p*-seed network: sampling, training, deployment
// ---------------------------------------------------------------------------
struct fc2d_b200_mlp {
    int device = 0;
    cudaStream_t st = nullptr;
    float *prm = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    void* blob = nullptr;
    float *partial = nullptr, *loss_partial = nullptr, *loss_dev = nullptr;
    int partial_blocks = 0;
    double* prim = nullptr;
    float *X = nullptr, *Y = nullptr, *Yp = nullptr;
    int *idx = nullptr, *iters = nullptr;
    int n = 0, cap = 0;
    int step = 0;
    double gamma = 1.4, tol = 1e-12;
    int tensor_form = 1;                 // batched evaluation: 1 tcgen05 tiles, 0 per-warp mma.sync
    unsigned* status = nullptr;          // STATUS_TENSOR of the tcgen05 evaluation (device)
};

// The network on n states: tcgen05 tiles of 128 states (default) or the per-warp form
// the solver uses.  The caller clears the status word first (mlp_clear) and checks it
// after synchronising the stream (mlp_status).
static void mlp_eval(fc2d_b200_mlp* m, const float* X, int n, float* Y)
{
    if (m->tensor_form) {
        launch_mlp_predict_tc(X, n, m->blob, Y, m->status, m->st);
    } else {
        launch_mlp_predict(X, n, m->blob, Y, m->st);
    }
}
static int mlp_clear(fc2d_b200_mlp* m)
{
    CK(cudaMemsetAsync(m->status, 0, sizeof(unsigned), m->st));
    return 0;
}
static int mlp_status(fc2d_b200_mlp* m)
{
    unsigned st = 0;
    CK(cudaMemcpy(&st, m->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (st & STATUS_TENSOR) return fail(FC2D_B200_EDEVICE, "device status: a tensor-core MMA of the network did not complete");
    return 0;
}

static unsigned long long host_splitmix(unsigned long long& s)
{
    unsigned long long z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static double host_uniform(unsigned long long& s) { return (double)(host_splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

static int mlp_partials(fc2d_b200_mlp* m, int nb)
{
    const int nblk = mlp_fwdbwd_blocks(nb);
    if (nblk <= m->partial_blocks) return 0;
    if (m->partial) cudaFree(m->partial);
    if (m->loss_partial) cudaFree(m->loss_partial);
    m->partial = nullptr; m->loss_partial = nullptr;
    CK(cudaMalloc(&m->partial, sizeof(float) * (size_t)nblk * MLP_NPARAM));
    CK(cudaMalloc(&m->loss_partial, sizeof(float) * (size_t)nblk));
    m->partial_blocks = nblk;
    return 0;
}

extern "C" int fc2d_b200_mlp_create(int device, unsigned long long seed, fc2d_b200_mlp_t** out)
{
    if (!out) return fail(FC2D_B200_EINVAL, "null argument");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(FC2D_B200_EDEVICE, "no such CUDA device");
    CK(cudaSetDevice(device));
    auto m = std::make_unique<fc2d_b200_mlp>();
    m->device = device;
    CK(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    CK(mlp_setup());
    CK(mlp_tc_setup());
    CK(cudaMalloc(&m->status, sizeof(unsigned)));
    CK(cudaMemset(m->status, 0, sizeof(unsigned)));
    CK(cudaMalloc(&m->prm, sizeof(float) * MLP_NPARAM));
    CK(cudaMalloc(&m->grad, sizeof(float) * MLP_NPARAM));
    CK(cudaMalloc(&m->m, sizeof(float) * MLP_NPARAM));
    CK(cudaMalloc(&m->v, sizeof(float) * MLP_NPARAM));
    CK(cudaMalloc(&m->blob, MLP_BLOB_BYTES));
    CK(cudaMalloc(&m->loss_dev, sizeof(float)));
    CK(cudaMemset(m->m, 0, sizeof(float) * MLP_NPARAM));
    CK(cudaMemset(m->v, 0, sizeof(float) * MLP_NPARAM));
    // Glorot-uniform weights, zero biases, from a splitmix64 stream of `seed`
    std::vector<float> p(MLP_NPARAM, 0.0f);
    unsigned long long s = seed;
    auto fill = [&](int off, int n, int fan_in, int fan_out) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for (int k = 0; k < n; k++) p[off + k] = (float)((2.0 * host_uniform(s) - 1.0) * a);
    };
    fill(MLP_OFF_W1, 64 * 6, 6, 64);
    fill(MLP_OFF_W2, 64 * 64, 64, 64);
    fill(MLP_OFF_W3, 64, 64, 1);
    CK(cudaMemcpy(m->prm, p.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice));
    launch_mlp_blob(m->prm, m->blob, m->st);
    CK(cudaStreamSynchronize(m->st));
    *out = m.release();
    return 0;
}

extern "C" int fc2d_b200_mlp_destroy(fc2d_b200_mlp_t* m)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m) return 0;
    cudaSetDevice(m->device);
    cudaStreamSynchronize(m->st);
    for (void* p : {(void*)m->prm, (void*)m->grad, (void*)m->m, (void*)m->v, m->blob, (void*)m->partial,
                    (void*)m->loss_partial, (void*)m->loss_dev, (void*)m->prim, (void*)m->X, (void*)m->Y,
                    (void*)m->Yp, (void*)m->idx, (void*)m->iters, (void*)m->status})
        if (p) cudaFree(p);
    cudaStreamDestroy(m->st);
    delete m;
    return 0;
}

extern "C" int fc2d_b200_mlp_set_params(fc2d_b200_mlp_t* m, const float* params)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m || !params) return fail(FC2D_B200_EINVAL, "null argument");
    CK(cudaSetDevice(m->device));
    CK(cudaMemcpyAsync(m->prm, params, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, m->st));
    launch_mlp_blob(m->prm, m->blob, m->st);
    CK(cudaStreamSynchronize(m->st));
    return 0;
}

extern "C" int fc2d_b200_mlp_get_params(fc2d_b200_mlp_t* m, float* params)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m || !params) return fail(FC2D_B200_EINVAL, "null argument");
    CK(cudaSetDevice(m->device));
    CK(cudaMemcpyAsync(params, m->prm, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return 0;
}

static int mlp_reserve(fc2d_b200_mlp* m, int n)
{
    if (n <= m->cap) return 0;
    for (void* p : {(void*)m->prim, (void*)m->X, (void*)m->Y, (void*)m->Yp, (void*)m->idx, (void*)m->iters})
        if (p) cudaFree(p);
    m->prim = nullptr; m->X = m->Y = m->Yp = nullptr; m->idx = m->iters = nullptr;
    CK(cudaMalloc(&m->prim, sizeof(double) * 6 * (size_t)n));
    CK(cudaMalloc(&m->X, sizeof(float) * MLP_IN * (size_t)n));
    CK(cudaMalloc(&m->Y, sizeof(float) * (size_t)n));
    CK(cudaMalloc(&m->Yp, sizeof(float) * (size_t)n));
    CK(cudaMalloc(&m->idx, sizeof(int) * (size_t)n));
    CK(cudaMalloc(&m->iters, sizeof(int) * (size_t)n));
    m->cap = n;
    return 0;
}

extern "C" int fc2d_b200_mlp_set_data(fc2d_b200_mlp_t* m, const double* prim, int n, double gamma, double tol)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m || !prim || n <= 0 || !(gamma > 1.0) || !(tol > 0.0)) return fail(FC2D_B200_EINVAL, "bad arguments");
    CK(cudaSetDevice(m->device));
    int rc = mlp_reserve(m, n);
    if (rc) return rc;
    CK(cudaMemcpyAsync(m->prim, prim, sizeof(double) * 6 * (size_t)n, cudaMemcpyHostToDevice, m->st));
    launch_mlp_targets(m->prim, n, gamma, tol, m->X, m->Y, m->iters, m->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(m->st));
    m->n = n; m->gamma = gamma; m->tol = tol;
    return 0;
}

extern "C" int fc2d_b200_mlp_get_data(fc2d_b200_mlp_t* m, float* X, float* Y)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m || m->n <= 0) return fail(FC2D_B200_ESTATE, "no training data");
    CK(cudaSetDevice(m->device));
    if (X) CK(cudaMemcpyAsync(X, m->X, sizeof(float) * MLP_IN * (size_t)m->n, cudaMemcpyDeviceToHost, m->st));
    if (Y) CK(cudaMemcpyAsync(Y, m->Y, sizeof(float) * (size_t)m->n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return 0;
}

extern "C" int fc2d_b200_mlp_train(fc2d_b200_mlp_t* m, int epochs, int batch, float lr, unsigned long long seed,
                                   double* loss_out)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m || m->n <= 0) return fail(FC2D_B200_ESTATE, "no training data");
    if (epochs <= 0 || batch <= 0 || !(lr > 0.0f)) return fail(FC2D_B200_EINVAL, "bad training arguments");
    CK(cudaSetDevice(m->device));
    const int n = m->n, nsteps = (n + batch - 1) / batch;
    int rc = mlp_partials(m, batch);
    if (rc) return rc;
    std::vector<int> perm(n);
    for (int i = 0; i < n; i++) perm[i] = i;
    unsigned long long s = seed;
    float* losses = nullptr;
    CK(cudaMalloc(&losses, sizeof(float) * (size_t)nsteps));
    double last = 0.0;
    for (int e = 0; e < epochs; e++) {
        for (int i = n - 1; i > 0; i--) {   // Fisher-Yates
            const int j = (int)(host_splitmix(s) % (unsigned long long)(i + 1));
            std::swap(perm[i], perm[j]);
        }
        CK(cudaMemcpyAsync(m->idx, perm.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, m->st));
        rc = mlp_clear(m);
        if (rc) return rc;
        for (int b = 0; b < nsteps; b++) {
            const int nb = std::min(batch, n - b * batch);
            m->step++;
            launch_mlp_step(m->X, m->Y, m->idx + (size_t)b * batch, nb, m->blob, m->prm, m->grad, m->m, m->v,
                            m->partial, m->loss_partial, losses + b, lr, m->step, true, m->status, m->st);
        }
        CK(cudaGetLastError());
        std::vector<float> l(nsteps);
        CK(cudaMemcpyAsync(l.data(), losses, sizeof(float) * nsteps, cudaMemcpyDeviceToHost, m->st));
        CK(cudaStreamSynchronize(m->st));
        double sum = 0.0;
        for (int b = 0; b < nsteps; b++) sum += l[b] * std::min(batch, n - b * batch);
        last = sum / n;
        rc = mlp_status(m);
        if (rc) { cudaFree(losses); return rc; }
    }
    cudaFree(losses);
    if (loss_out) *loss_out = last;
    return 0;
}

extern "C" int fc2d_b200_mlp_gradient(fc2d_b200_mlp_t* m, const float* X, const float* Y, int n, float* grad,
                                      double* loss)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m || !X || !Y || !grad || n <= 0) return fail(FC2D_B200_EINVAL, "bad arguments");
    CK(cudaSetDevice(m->device));
    int rc = mlp_partials(m, n);
    if (rc) return rc;
    float *Xd, *Yd;
    CK(cudaMalloc(&Xd, sizeof(float) * MLP_IN * (size_t)n));
    CK(cudaMalloc(&Yd, sizeof(float) * (size_t)n));
    CK(cudaMemcpyAsync(Xd, X, sizeof(float) * MLP_IN * (size_t)n, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(Yd, Y, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, m->st));
    rc = mlp_clear(m);
    if (rc) return rc;
    launch_mlp_step(Xd, Yd, nullptr, n, m->blob, m->prm, m->grad, m->m, m->v, m->partial, m->loss_partial,
                    m->loss_dev, 0.0f, 1, false, m->status, m->st);
    float l = 0.0f;
    CK(cudaMemcpyAsync(grad, m->grad, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, m->st));
    CK(cudaMemcpyAsync(&l, m->loss_dev, sizeof(float), cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    cudaFree(Xd); cudaFree(Yd);
    if (loss) *loss = l;
    return mlp_status(m);
}

extern "C" int fc2d_b200_mlp_predict(fc2d_b200_mlp_t* m, const float* X, int n, float* Y)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m || !X || !Y || n <= 0) return fail(FC2D_B200_EINVAL, "bad arguments");
    CK(cudaSetDevice(m->device));
    float *Xd, *Yd;
    CK(cudaMalloc(&Xd, sizeof(float) * MLP_IN * (size_t)n));
    CK(cudaMalloc(&Yd, sizeof(float) * (size_t)n));
    CK(cudaMemcpyAsync(Xd, X, sizeof(float) * MLP_IN * (size_t)n, cudaMemcpyHostToDevice, m->st));
    int rc = mlp_clear(m);
    if (rc) return rc;
    mlp_eval(m, Xd, n, Yd);
    CK(cudaMemcpyAsync(Y, Yd, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    cudaFree(Xd); cudaFree(Yd);
    return mlp_status(m);
}

extern "C" int fc2d_b200_mlp_newton_histogram(fc2d_b200_mlp_t* m, int use_mlp, long long* hist)
{
    DeviceScope dev_scope_(m ? m->device : -1);
    if (!m || !hist || m->n <= 0) return fail(FC2D_B200_ESTATE, "no data");
    CK(cudaSetDevice(m->device));
    if (use_mlp) {
        const int rc = mlp_clear(m);
        if (rc) return rc;
        mlp_eval(m, m->X, m->n, m->Yp);
    }
    launch_mlp_newton_iters(m->prim, m->X, use_mlp ? m->Yp : nullptr, m->n, m->gamma, m->tol, m->iters, m->st);
    std::vector<int> it(m->n);
    CK(cudaMemcpyAsync(it.data(), m->iters, sizeof(int) * (size_t)m->n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    if (use_mlp) {
        const int rc = mlp_status(m);
        if (rc) return rc;
    }
    for (int k = 0; k < 32; k++) hist[k] = 0;
    for (int v : it) hist[v < 31 ? v : 31]++;
    return 0;
}

extern "C" int fc2d_b200_mlp_set_tensor_form(fc2d_b200_mlp_t* m, int tcgen05)
{
    if (!m) return fail(FC2D_B200_EINVAL, "null network");
    m->tensor_form = tcgen05 != 0;
    return 0;
}

extern "C" int fc2d_b200_sample_interfaces(fc2d_b200_solver_t* s, int n, unsigned long long seed, double* prim)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized || !prim || n <= 0) return fail(FC2D_B200_EINVAL, "bad arguments");
    if (s->o.rp != FC2D_B200_RP_EULER_EXACT) return fail(FC2D_B200_EINVAL, "interface sampling needs the Euler solver");
    double* d = nullptr;
    CK(cudaMalloc(&d, sizeof(double) * 6 * (size_t)n));
    launch_sample_interfaces(s->d, s->q, s->forest.np(), s->o.gamma, seed, n, d, s->st);
    cudaError_t e = cudaMemcpyAsync(prim, d, sizeof(double) * 6 * (size_t)n, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(d);
    if (e != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("sample_interfaces: ") + cudaGetErrorString(e));
    return 0;
}

extern "C" int fc2d_b200_set_pstar_seed(fc2d_b200_solver_t* s, const fc2d_b200_mlp_t* m)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    if (!m) { s->use_mlp = false; return 0; }
    if (s->o.rp != FC2D_B200_RP_EULER_EXACT) return fail(FC2D_B200_EINVAL, "the p* seed applies to the Euler solver");
    if (!s->mlp_blob) CK(cudaMalloc(&s->mlp_blob, MLP_BLOB_BYTES));
    CK(cudaMemcpyAsync(s->mlp_blob, m->blob, MLP_BLOB_BYTES, cudaMemcpyDeviceToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->use_mlp = true;
    return 0;
}

// ---------------------------------------------------------------------------
// batches of independent forests
// ---------------------------------------------------------------------------
extern "C" int fc2d_b200_set_instances(fc2d_b200_solver_t* s, int n, const fc2d_b200_instance_t* inst)
{
    DeviceScope dev_scope_(s);
    if (s && s->part) return fail(FC2D_B200_EINVAL, "a partitioned solver holds one forest");
    if (!s || n <= 0 || !inst) return fail(FC2D_B200_EINVAL, "bad arguments");
    if (n > FC2D_B200_MAX_INSTANCES) return fail(FC2D_B200_EINVAL, "too many instances");
    if (s->initialized) return fail(FC2D_B200_ESTATE, "instances are set before initialize");
    if (s->o.app == FC2D_B200_APP_SWIRL)
        return fail(FC2D_B200_EINVAL, "batched instances need a time-independent app (the swirl velocity depends on t)");
    int span = 0;
    std::vector<Geometry> G(n);
    for (int i = 0; i < n; i++) {
        const fc2d_b200_instance_t& I = inst[i];
        if (I.minlevel < 0 || I.maxlevel < I.minlevel || I.maxlevel > 20 || I.mi <= 0 || I.mj <= 0)
            return fail(FC2D_B200_EINVAL, "bad instance levels or brick");
        span = std::max(span, I.maxlevel - I.minlevel);
        G[i] = Geometry{s->d, I.mi, I.mj, I.ax, I.bx, I.ay, I.by, I.minlevel};
    }
    s->insts.assign(inst, inst + n);
    s->forest.inst = G;
    s->forest.g = G[0];
    s->o.minlevel = 0;
    s->o.maxlevel = span;
    s->ncfl = n;
    invalidate_graph(s);
    return 0;
}

extern "C" int fc2d_b200_num_instances(const fc2d_b200_solver_t* s, int* n)
{
    if (!s || !n) return fail(FC2D_B200_EINVAL, "null argument");
    *n = s->forest.ninst();
    return 0;
}

extern "C" int fc2d_b200_patch_instance(const fc2d_b200_solver_t* s, int* inst)
{
    if (!s || !inst) return fail(FC2D_B200_EINVAL, "null argument");
    for (int i = 0; i < s->forest.np(); i++) inst[i] = s->forest.p[i].inst;
    return 0;
}

extern "C" int fc2d_b200_advance_instances_begin(fc2d_b200_solver_t* s, const double* dt)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized || !dt) return fail(FC2D_B200_EINVAL, "bad arguments");
    if (s->insts.empty()) return fail(FC2D_B200_ESTATE, "no instances set");
    if (s->pending) return fail(FC2D_B200_ESTATE, "an advance is in flight");
    const int n = (int)s->insts.size();
    for (int i = 0; i < n; i++)
        if (!(dt[i] > 0.0)) return fail(FC2D_B200_EINVAL, "instance time steps must be positive");
    std::memcpy(s->inst_dt_host, dt, sizeof(double) * n);
    CK(cudaMemcpyAsync(s->inst_dt_dev, s->inst_dt_host, sizeof(double) * n, cudaMemcpyHostToDevice, s->st));
    // the level time steps 2^-l of a unit coarse step scale each instance's own dt
    return advance_launch(s, 0.0, 1.0);
}

extern "C" int fc2d_b200_advance_instances_end(fc2d_b200_solver_t* s, double* cfl)
{
    DeviceScope dev_scope_(s);
    if (!s) return fail(FC2D_B200_EINVAL, "null solver");
    double dummy = 0.0;
    return advance_finish(s, &dummy, cfl);
}

extern "C" int fc2d_b200_advance_instances(fc2d_b200_solver_t* s, const double* dt, double* cfl)
{
    DeviceScope dev_scope_(s);
    int rc = fc2d_b200_advance_instances_begin(s, dt);
    if (rc) return rc;
    return fc2d_b200_advance_instances_end(s, cfl);
}

extern "C" int fc2d_b200_mass_instances(fc2d_b200_solver_t* s, double* out)
{
    DeviceScope dev_scope_(s);
    if (!s || !out || !s->initialized) return fail(FC2D_B200_EINVAL, "bad arguments");
    const int np = s->forest.np(), meqn = s->d.meqn, ni = s->forest.ninst();
    if (np * meqn > s->mass_cap) {
        if (s->mass_dev) cudaFree(s->mass_dev);
        s->mass_cap = np * meqn + 1024;
        CK(cudaMalloc(&s->mass_dev, sizeof(double) * (size_t)s->mass_cap));
    }
    launch_patch_mass(s->d, s->q, s->desc, np, s->mass_dev, s->st, s->area);
    std::vector<double> pm((size_t)np * meqn);
    CK(cudaMemcpyAsync(pm.data(), s->mass_dev, sizeof(double) * pm.size(), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    std::vector<double> sum((size_t)ni * meqn, 0.0), comp((size_t)ni * meqn, 0.0);
    for (int p = 0; p < np; p++) {
        const int i = s->forest.p[p].inst;
        for (int m = 0; m < meqn; m++) {
            double& S = sum[(size_t)i * meqn + m];
            double& C = comp[(size_t)i * meqn + m];
            const double y = pm[(size_t)p * meqn + m] - C;
            const double t = S + y;
            C = (t - S) - y;
            S = t;
        }
    }
    for (size_t k = 0; k < sum.size(); k++) out[k] = sum[k];
    return 0;
}

// ---------------------------------------------------------------------------
// patch-to-CTA variants and the autotuner
// ---------------------------------------------------------------------------
extern "C" int fc2d_b200_num_variants(const fc2d_b200_solver_t* s, int* n, int* current)
{
    if (!s || !n) return fail(FC2D_B200_EINVAL, "null argument");
    *n = (int)s->vars.size();
    if (current) *current = s->var;
    return 0;
}

extern "C" int fc2d_b200_variant_info(const fc2d_b200_solver_t* s, int v, int* threads, int* min_blocks, int* reg,
                                      int* smem_bytes, int* persistent)
{
    if (!s || v < 0 || v >= (int)s->vars.size()) return fail(FC2D_B200_EINVAL, "no such variant");
    const Step2Variant* x = s->vars[v];
    if (threads) *threads = x->threads;
    if (min_blocks) *min_blocks = x->min_blocks;
    if (reg) *reg = x->reg;
    if (smem_bytes) *smem_bytes = x->smem;
    if (persistent) *persistent = x->persistent;
    return 0;
}

extern "C" int fc2d_b200_set_variant(fc2d_b200_solver_t* s, int v)
{
    DeviceScope dev_scope_(s);
    if (!s || v < 0 || v >= (int)s->vars.size()) return fail(FC2D_B200_EINVAL, "no such variant");
    cudaError_t e = s->vars[v]->fn(nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0, nullptr, LevelGroup{1, {0}}, nullptr, s->st);
    if (e != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("kernel setup: ") + cudaGetErrorString(e));
    s->var = v;
    for (int l = 0; l < 33; l++) s->var_lev[l] = -1;
    invalidate_graph(s);
    return 0;
}

// Time every variant on the current forest -- one launch per level, as a
// subcycled step issues them -- and keep the fastest.  The timed launches run
// with dt = 0 and neither store fluxes, accumulate waves, save q nor count
// Newton iterations, so they do all of the update's arithmetic but leave q,
// the registers and the statistics as they were.
extern "C" int fc2d_b200_autotune(fc2d_b200_solver_t* s, int reps, int* best_out, double* ms_out)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized || reps < 1) return fail(FC2D_B200_EINVAL, "bad arguments");
    const Forest& f = s->forest;
    StepParams sp = make_params(s, f.maxlevel_present, s->t_curr, 0.0);
    sp.store_flux = 0; sp.accumulate_waves = 0; sp.save_last = 0; sp.newton_hist = nullptr;
    CK(cudaMemcpyAsync(s->tune_params, &sp, sizeof(StepParams), cudaMemcpyHostToDevice, s->st));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto pass = [&](const Step2Variant* v) -> cudaError_t {
        for (int l = 0; l <= 32; l++) {
            const int p0 = f.lev_off[l], np = f.lev_off[l + 1] - p0;
            if (np <= 0) continue;
            cudaError_t e = v->fn(s->q, s->qlast, s->aux, s->regs, s->desc, p0, np, s->tune_params, LevelGroup{1, {0}}, s->cfl_dev, s->st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    int best = s->var;
    double best_ms = 1e300;
    cudaError_t err = cudaSuccess;
    for (int v = 0; v < (int)s->vars.size() && err == cudaSuccess; v++) {
        err = s->vars[v]->fn(nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0, nullptr, LevelGroup{1, {0}}, nullptr, s->st);
        if (err == cudaSuccess) err = pass(s->vars[v]);             // warm-up
        if (err == cudaSuccess) err = cudaEventRecord(e0, s->st);
        for (int r = 0; r < reps && err == cudaSuccess; r++) err = pass(s->vars[v]);
        if (err == cudaSuccess) err = cudaEventRecord(e1, s->st);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        const double per = (double)ms / reps;
        if (ms_out) ms_out[v] = per;
        if (err == cudaSuccess && per < best_ms) { best_ms = per; best = v; }
    }
    // then per level: a level's patch count decides how its CTAs fill the waves
    // of the device, so a level takes another variant where that is clearly faster
    // on it alone (by 5 %: the forest changes between regrids, and a small level's
    // launch is a few microseconds); each level's timing covers at least ~0.3 ms
    auto time_level = [&](const Step2Variant* x, int p0, int np, int n, double& per) -> cudaError_t {
        cudaError_t e = x->fn(s->q, s->qlast, s->aux, s->regs, s->desc, p0, np, s->tune_params, LevelGroup{1, {0}}, s->cfl_dev, s->st);
        if (e == cudaSuccess) e = cudaEventRecord(e0, s->st);
        for (int r = 0; r < n && e == cudaSuccess; r++)
            e = x->fn(s->q, s->qlast, s->aux, s->regs, s->desc, p0, np, s->tune_params, LevelGroup{1, {0}}, s->cfl_dev, s->st);
        if (e == cudaSuccess) e = cudaEventRecord(e1, s->st);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        per = (double)ms / n;
        return e;
    };
    int lev_best[33];
    for (int l = 0; l <= 32 && err == cudaSuccess; l++) {
        lev_best[l] = -1;
        const int p0 = f.lev_off[l], np = f.lev_off[l + 1] - p0;
        if (np <= 0) continue;
        double est = 0.0, ref = 0.0;
        err = time_level(s->vars[best], p0, np, 1, est);
        const int n = std::max(reps, std::min(64, (int)(0.3 / std::max(est, 1e-3))));
        if (err == cudaSuccess) err = time_level(s->vars[best], p0, np, n, ref);
        lev_best[l] = best;
        double lbest = 0.95 * ref;
        for (int v = 0; v < (int)s->vars.size() && err == cudaSuccess; v++) {
            if (v == best) continue;
            double per = 0.0;
            err = time_level(s->vars[v], p0, np, n, per);
            if (err == cudaSuccess && per < lbest) { lbest = per; lev_best[l] = v; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("autotune: ") + cudaGetErrorString(err));
    s->var = best;
    for (int l = 0; l < 33; l++) s->var_lev[l] = lev_best[l];
    invalidate_graph(s);
    if (best_out) *best_out = best;
    return 0;
}

extern "C" int fc2d_b200_level_variants(const fc2d_b200_solver_t* s, int* variant)
{
    if (!s || !variant) return fail(FC2D_B200_EINVAL, "bad arguments");
    for (int l = 0; l < 33; l++) variant[l] = s->var_lev[l] >= 0 ? s->var_lev[l] : s->var;
    return 0;
}

// A per-level choice made earlier (fc2d_b200_level_variants of a tuned solver of the
// same shape) applied without timing anything.
extern "C" int fc2d_b200_set_level_variants(fc2d_b200_solver_t* s, const int* variant)
{
    DeviceScope dev_scope_(s);
    if (!s || !variant) return fail(FC2D_B200_EINVAL, "bad arguments");
    for (int l = 0; l < 33; l++)
        if (variant[l] < 0 || variant[l] >= (int)s->vars.size())
            return fail(FC2D_B200_EINVAL, "no such variant for level " + std::to_string(l));
    for (int l = 0; l < 33; l++) {
        bool seen = false;
        for (int k = 0; k < l; k++) seen = seen || variant[k] == variant[l];
        if (seen) continue;
        cudaError_t e = s->vars[variant[l]]->fn(nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0, nullptr,
                                                LevelGroup{1, {0}}, nullptr, s->st);
        if (e != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("kernel setup: ") + cudaGetErrorString(e));
    }
    for (int l = 0; l < 33; l++) s->var_lev[l] = variant[l];
    invalidate_graph(s);
    return 0;
}

// ---------------------------------------------------------------------------
// output (fclaw2d_clawpatch_output_ascii)
// ---------------------------------------------------------------------------
extern "C" int fc2d_b200_output_ascii(fc2d_b200_solver_t* s, const char* dir, int iframe, double time)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized || !dir) return fail(FC2D_B200_EINVAL, "bad arguments");
    const Forest& f = s->forest;
    const int np = f.np();
    const size_t nq = (size_t)s->d.nq();
    std::vector<double> q((size_t)np * nq);
    CK(cudaMemcpyAsync(q.data(), s->q, q.size() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    // the reference writes patches block by block, each block's leaves along the curve
    std::vector<int> order(np);
    for (int i = 0; i < np; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const PatchInfo& A = f.p[a];
        const PatchInfo& B = f.p[b];
        if (A.inst != B.inst) return A.inst < B.inst;
        if (A.block != B.block) return A.block < B.block;
        return A.morton < B.morton;
    });
    std::vector<int> lev(np), blk(np);
    std::vector<double> xl(np), yl(np), dx(np), dy(np), qo((size_t)np * nq);
    for (int k = 0; k < np; k++) {
        const PatchInfo& P = f.p[order[k]];
        lev[k] = P.level + f.gi(P.inst).lbase;
        blk[k] = P.block;
        xl[k] = P.xlower; yl[k] = P.ylower; dx[k] = P.dx; dy[k] = P.dy;
        std::memcpy(&qo[(size_t)k * nq], &q[(size_t)order[k] * nq], nq * sizeof(double));
    }
    const int rc = fc2d_b200_write_ascii_frame(dir, iframe, time, s->d.meqn, s->d.maux, s->d.mx, s->d.my, s->d.mbc, np,
                                               lev.data(), blk.data(), xl.data(), yl.data(), dx.data(), dy.data(),
                                               qo.data());
    if (rc) return fail(rc, std::string("cannot write fort.q/fort.t frame into ") + dir);
    return 0;
}

// fclaw2d_clawpatch_output_vtk (src/patches/clawpatch/fclaw2d_clawpatch_output_vtk.c:880-900):
// <prefix>_frame_NNNN.vtu.  The device packs points and cell values of every patch
// in the file's patch order (block by block, each block's leaves along the curve);
// one copy brings them to the host, which writes the file.
extern "C" int fc2d_b200_output_vtk(fc2d_b200_solver_t* s, const char* prefix, int iframe)
{
    DeviceScope dev_scope_(s);
    if (!s || !s->initialized || !prefix || iframe < 0) return fail(FC2D_B200_EINVAL, "bad arguments");
    const Forest& f = s->forest;
    const int np = f.np();
    std::vector<int> order(np);
    for (int i = 0; i < np; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const PatchInfo& A = f.p[a];
        const PatchInfo& B = f.p[b];
        if (A.inst != B.inst) return A.inst < B.inst;
        if (A.block != B.block) return A.block < B.block;
        return A.morton < B.morton;
    });
    std::vector<int> blk(np);
    for (int k = 0; k < np; k++) blk[k] = f.p[order[k]].block;
    const size_t npt = (size_t)(s->d.mx + 1) * (s->d.my + 1), ncell = (size_t)s->d.mx * s->d.my;
    std::vector<double> pts((size_t)np * npt * 3);
    std::vector<float> vals((size_t)np * ncell * s->d.meqn);
    int* ord_d = nullptr;
    double* pts_d = nullptr;
    float* vals_d = nullptr;
    cudaError_t e = cudaMalloc(&ord_d, sizeof(int) * (np > 0 ? np : 1));
    if (e == cudaSuccess) e = cudaMalloc(&pts_d, sizeof(double) * (pts.size() > 0 ? pts.size() : 1));
    if (e == cudaSuccess) e = cudaMalloc(&vals_d, sizeof(float) * (vals.size() > 0 ? vals.size() : 1));
    if (e == cudaSuccess && np > 0)
        e = cudaMemcpyAsync(ord_d, order.data(), sizeof(int) * np, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) {
        launch_vtk_pack(s->d, s->q, s->desc, ord_d, np, s->sphere ? 1 : 0, pts_d, vals_d, s->st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && np > 0)
        e = cudaMemcpyAsync(pts.data(), pts_d, sizeof(double) * pts.size(), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess && np > 0)
        e = cudaMemcpyAsync(vals.data(), vals_d, sizeof(float) * vals.size(), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (ord_d) cudaFree(ord_d);
    if (pts_d) cudaFree(pts_d);
    if (vals_d) cudaFree(vals_d);
    if (e != cudaSuccess) return fail(FC2D_B200_ECUDA, std::string("vtk output: ") + cudaGetErrorString(e));
    char name[64];
    std::snprintf(name, sizeof(name), "_frame_%04d.vtu", iframe);
    const std::string path = std::string(prefix) + name;
    const int rc = fc2d_b200_write_vtk_file(path.c_str(), s->d.mx, s->d.my, s->d.meqn, np, blk.data(), pts.data(),
                                            vals.data());
    if (rc) return fail(rc, "cannot write " + path);
    return 0;
}
