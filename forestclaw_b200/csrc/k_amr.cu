// k_amr.cu -- ghost-fill, time-sync, diagnostics and regrid kernels.
//
// Ghost fill runs from gather tables built on the host at regrid time: every
// ghost cell the reference's copy / average / interpolate / physical-BC
// callbacks would write in one stage becomes one table entry (last writer of the
// reference's callback order wins), so each stage is one launch with one thread
// per ghost cell and disjoint destinations.  Arithmetic follows the clawpatch
// 4.6 Fortran in evaluation order; this file is compiled without FMA
// contraction so the FP64 results match the FP64 CPU path bit for bit.
//   average face/corner   fort_4.6/fclaw2d_clawpatch46_average.f:16-272
//   interpolate           fort_4.6/fclaw2d_clawpatch46_interpolate.f:30-392, utils.f:45-63
//   physical BC           clawpack46_bc2_default.f:1-213
//   timeinterp            fort_4.6/fclaw2d_clawpatch46_timeinterp.f:11-78
//   time sync             clawpack46_time_sync.f:254-704, clawpatch_conservation.c:207-280
//   mass                  fort_4.6/fclaw2d_clawpatch46_diagnostics.f:13-55
//   tagging               fort_4.6/fclaw2d_clawpatch46_tag4refinement.f / _tag4coarsening.f
#include "fcb_launch.cuh"
#include "kernels.h"

namespace fcb {

static thread_local bool tl_programmatic = false;
void set_programmatic_launch(bool on) { tl_programmatic = on; }
bool programmatic_launch() { return tl_programmatic; }

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

// The gather stages take up to two table segments, each with its own arrays:
// a ghost-fill stage on q and the same stage on the time-interpolated copy
// write different arrays and read cells the other does not write, so they
// share a launch.  Interpolation and physical BCs: one thread per (entry, field),
// segment 0's threads first, field-major within a segment, so a warp handles
// consecutive entries of one field (the fields of an entry are independent).
template <class E>
__device__ __forceinline__ bool seg_item(const GatherSeg<E>& s0, const GatherSeg<E>& s1, int meqn, long t,
                                         GatherSeg<E>& g, int& e, int& m)
{
    const long n0 = (long)s0.n * meqn;
    if (t < n0) {
        g = s0;
    } else {
        t -= n0;
        g = s1;
    }
    if (t >= (long)g.n * meqn) return false;
    m = (int)(t / g.n);
    e = (int)(t - (long)m * g.n);
    return true;
}
__device__ __forceinline__ long flat_index() { return (long)blockIdx.x * blockDim.x + threadIdx.x; }

// Patch shape of the region-op index arithmetic: compile-time for the common square
// patches with mbc 2 (the divisions by mbc and mx become shifts), run-time otherwise.
template <int MX, int MBC>
struct FixedShape {
    static constexpr int mx = MX, my = MX, mbc = MBC;
    __device__ FixedShape(int, int, int) {}
};
struct RunShape {
    int mx, my, mbc;
    __device__ RunShape(int mx_, int my_, int mbc_) : mx(mx_), my(my_), mbc(mbc_) {}
};

// Fortran cell (i, j) of the k-th ghost cell of a region op (FillOp): faces row by row
// with i fastest, corners likewise; the cells a region covers, below.
template <class S>
__device__ __forceinline__ int region_cells(const S& P, int region)
{
    return region < 2 ? P.mbc * P.my : (region < 4 ? P.mx * P.mbc : P.mbc * P.mbc);
}
template <class S>
__device__ __forceinline__ void region_cell(const S& P, int region, int k, int& i, int& j)
{
    if (region < 2) {
        i = (region == 0 ? 1 - P.mbc : P.mx + 1) + k % P.mbc;
        j = 1 + k / P.mbc;
    } else if (region < 4) {
        i = 1 + k % P.mx;
        j = (region == 2 ? 1 - P.mbc : P.my + 1) + k / P.mx;
    } else {
        const int cr = region - 4;
        i = ((cr & 1) ? P.mx + 1 : 1 - P.mbc) + k % P.mbc;
        j = ((cr & 2) ? P.my + 1 : 1 - P.mbc) + k / P.mbc;
    }
}

// One ghost cell of a copy op, every field: the fields are read before any is written.
template <class S>
__device__ __forceinline__ void copy_cell(const S& P, const GatherSeg<FillOp>& g, int o, int k, int meqn)
{
    const FillOp op = g.e[o];
    if (k >= region_cells(P, op.region)) return;
    const int nx = P.mx + 2 * P.mbc, nxy = nx * (P.my + 2 * P.mbc);
    int i, j;
    region_cell(P, op.region, k, i, j);
    const int i2 = op.ci + op.ii * i + op.ij * j, j2 = op.cj + op.ji * i + op.jj * j;
    const long nq = (long)nxy * meqn;
    double* d = g.dst + op.dst * nq + (j + P.mbc - 1) * nx + (i + P.mbc - 1);
    const double* s = g.src + op.src * nq + (j2 + P.mbc - 1) * nx + (i2 + P.mbc - 1);
    for (int m0 = 0; m0 < meqn; m0 += 4) {
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (m0 + u < meqn) v[u] = s[(m0 + u) * nxy];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (m0 + u < meqn) d[(m0 + u) * nxy] = v[u];
    }
}

// One coarse ghost cell of an average op, every field: the mean of its four children
// (fine cells at (0,0), (1,0), (0,1), (1,1) of the coarse cell's own axes), in that order.
template <bool AREA, class S>
__device__ __forceinline__ void average_cell(const S& P, const GatherSeg<FillOp>& g, int o, int k, int meqn,
                                             const double* __restrict__ area)
{
    const FillOp op = g.e[o];
    if (k >= region_cells(P, op.region)) return;
    const int nx = P.mx + 2 * P.mbc, nxy = nx * (P.my + 2 * P.mbc);
    int ic, jc;
    region_cell(P, op.region, k, ic, jc);
    // children (0,0), (1,0), (0,1), (1,1) of (ic, jc) at (i0, j0), + (ii, ji), + (ij, jj)
    // and + both: the map is an isometry, so the extremes of their indices are these sums
    const int i0 = op.ci + op.ii * (2 * ic) + op.ij * (2 * jc), j0 = op.cj + op.ji * (2 * ic) + op.jj * (2 * jc);
    if (op.region < 4) {
        // a face keeps the coarse cells whose children are all interior fine cells
        const int ilo = i0 + min(op.ii, 0) + min(op.ij, 0), ihi = i0 + max(op.ii, 0) + max(op.ij, 0);
        const int jlo = j0 + min(op.ji, 0) + min(op.jj, 0), jhi = j0 + max(op.ji, 0) + max(op.jj, 0);
        if (ilo < 1 || ihi > P.mx || jlo < 1 || jhi > P.my) return;
    }
    const int c0 = (j0 + P.mbc - 1) * nx + (i0 + P.mbc - 1);   // child (0,0): plane-0 offset in the fine patch
    const int o1 = op.ii + op.ji * nx, o2 = op.ij + op.jj * nx, o3 = o1 + o2;
    const long nq = (long)nxy * meqn;
    double* __restrict__ d = g.dst + op.dst * nq + (jc + P.mbc - 1) * nx + (ic + P.mbc - 1);
    const double* __restrict__ src = g.src + op.src * nq + c0;
    if constexpr (AREA) {
        // manifold (fclaw2d_clawpatch46_average.f:96-115): sum(q_f a_f) / sum(a_f); the
        // area array of a patch has one ring more than q: cell (ic, jc) of q's padded
        // layout is (ic + 1, jc + 1) of a row of nx + 2
        const int na = (nx + 2) * (P.my + 2 * P.mbc + 2);
        const double* ap = area + (size_t)op.src * na;
        auto ai = [&](int off) { const int c = c0 + off; return (c / nx + 1) * (nx + 2) + c % nx + 1; };
        const double a0 = ap[ai(0)], a1 = ap[ai(o1)], a2 = ap[ai(o2)], a3 = ap[ai(o3)];
        for (int m = 0; m < meqn; m++) {
            const double* f = src + m * nxy;
            double sum = 0.0, af = 0.0;
            sum = sum + f[0] * a0;  af = af + a0;
            sum = sum + f[o1] * a1; af = af + a1;
            sum = sum + f[o2] * a2; af = af + a2;
            sum = sum + f[o3] * a3; af = af + a3;
            d[m * nxy] = sum / af;
        }
        return;
    }
    for (int m = 0; m < meqn; m++) {
        const double* f = src + m * nxy;
        double sum = 0.0;
        sum = sum + f[0];
        sum = sum + f[o1];
        sum = sum + f[o2];
        sum = sum + f[o3];
        d[m * nxy] = sum / 4.0;
    }
}

// thread t of two op segments of `slot` threads per op: segment (by value: the
// parameters stay in the constant bank), op, cell
__device__ __forceinline__ bool op_index(const GatherSeg<FillOp>& s0, const GatherSeg<FillOp>& s1, int slot, long t,
                                         GatherSeg<FillOp>& g, int& o, int& k)
{
    const long n0 = (long)s0.n * slot;
    const bool second = t >= n0;
    if (second) t -= n0;
    g.dst = second ? s1.dst : s0.dst;
    g.src = second ? s1.src : s0.src;
    g.e = second ? s1.e : s0.e;
    g.n = second ? s1.n : s0.n;
    if (t >= (long)g.n * slot) return false;
    o = (int)(t / slot);
    k = (int)(t - (long)o * slot);
    return true;
}

// The average and copy stages of one ghost update in one launch: averaging writes
// the ghost cells a coarse patch has beside finer neighbours, copying those beside
// same-size neighbours (disjoint cells), and both read interior cells only, which
// neither writes.  One thread per (op, cell) with mbc * max(mx, my) threads per op
// (a face's cells; a corner uses mbc * mbc of them); the average segments first.
// AREA: the area-weighted average of a manifold (cell areas in `area`).
template <class S, bool AREA>
__global__ void __launch_bounds__(256, AREA ? 4 : 8)
k_average_copy(GatherSeg<FillOp> a0, GatherSeg<FillOp> a1, GatherSeg<FillOp> c0, GatherSeg<FillOp> c1, int mx,
               int my, int mbc, int meqn, const double* __restrict__ area)
{
    grid_dependency_wait();       // programmatic launch: the previous grid's writes are visible
    grid_launch_dependents();
    const S P(mx, my, mbc);
    const int slot = P.mbc * (P.mx > P.my ? P.mx : P.my);
    const long t = flat_index();
    const long na = ((long)a0.n + a1.n) * slot;
    GatherSeg<FillOp> g;
    int o, k;
    if (t < na) {
        if (op_index(a0, a1, slot, t, g, o, k)) average_cell<AREA>(P, g, o, k, meqn, area);
    } else if (op_index(c0, c1, slot, t - na, g, o, k)) {
        copy_cell(P, g, o, k, meqn);
    }
}

// AMRClaw limited slopes (fclaw2d_clawpatch_utils.f:52-55, mth = 5)
__device__ __forceinline__ double compute_slopes(double sl, double sr)
{
    double sc = (sl + sr) / 2.0;
    double a = fabs(sl) * 2.0, b = fabs(sr) * 2.0, c = fabs(sc);
    double mn = a < b ? a : b;
    mn = mn < c ? mn : c;
    double s = copysign(1.0, sl * sr);
    return mn * (s > 0.0 ? s : 0.0) * copysign(1.0, sc);
}

__device__ __forceinline__ void interp_at(const GatherSeg<InterpEnt>& s0, const GatherSeg<InterpEnt>& s1, long t,
                                          int nx, int nxy, int meqn)
{
    GatherSeg<InterpEnt> g;
    int e, m;
    if (!seg_item(s0, s1, meqn, t, g, e, m)) return;
    double* __restrict__ dst = g.dst;
    const double* __restrict__ src = g.src;
    const InterpEnt c = g.e[e];
    const double shx = (c.sub & 1) ? 0.25 : -0.25;
    const double shy = (c.sub & 2) ? 0.25 : -0.25;
    const double* qc = src + c.src + m * nxy;
    double q0 = qc[0];
    double sl = (q0 - qc[-1]);
    double sr = (qc[1] - q0);
    double gradx = compute_slopes(sl, sr);
    sl = (q0 - qc[-nx]);
    sr = (qc[nx] - q0);
    double grady = compute_slopes(sl, sr);
    dst[c.dst + m * nxy] = q0 + gradx * shx + grady * shy;
}
__global__ void k_interp(GatherSeg<InterpEnt> s0, GatherSeg<InterpEnt> s1, int nx, int nxy, int meqn)
{
    grid_dependency_wait();       // programmatic launch: the previous grid's writes are visible
    grid_launch_dependents();
    interp_at(s0, s1, flat_index(), nx, nxy, meqn);
}

__device__ __forceinline__ void phys_at(const GatherSeg<PhysEnt>& s0, const GatherSeg<PhysEnt>& s1, long t, int nxy,
                                        int meqn, const double* __restrict__ bcstate)
{
    GatherSeg<PhysEnt> g;
    int e, m;
    if (!seg_item(s0, s1, meqn, t, g, e, m)) return;
    double* __restrict__ q = g.dst;                 // in place: sources are cells of the same array
    const PhysEnt c = g.e[e];
    const double v = c.cst ? bcstate[m] : q[c.src + m * nxy];
    q[c.dst + m * nxy] = ((c.neg >> m) & 1) ? -v : v;
}
__global__ void k_phys(GatherSeg<PhysEnt> s0, GatherSeg<PhysEnt> s1, int nxy, int meqn,
                       const double* __restrict__ bcstate)
{
    grid_dependency_wait();       // programmatic launch: the previous grid's writes are visible
    grid_launch_dependents();
    phys_at(s0, s1, flat_index(), nxy, meqn, bcstate);
}

// Band of width mbc inside the patch, in the four loops of timeinterp.f:33-70: one
// index per (listed patch, cell of the padded patch); a stage may cover the lists
// of several levels, each with its own alpha (alpha.a[level]).
__device__ __forceinline__ void timeinterp_at(const double* __restrict__ q, const double* __restrict__ ql,
                                              double* __restrict__ qi, const int* __restrict__ patches,
                                              const PatchDesc* __restrict__ desc, int mx, int my, int mbc, int meqn,
                                              const LevelAlpha& la, long t)
{
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc, nxy = nx * ny;
    const int pi = (int)(t / nxy), c = (int)(t - (long)pi * nxy);
    const int ic = c % nx, jc = c / nx;
    const int i = ic - mbc + 1, j = jc - mbc + 1;         // Fortran indices
    if (i < 1 || i > mx || j < 1 || j > my) return;
    const bool band = (i <= mbc) || (i > mx - mbc) || (j <= mbc) || (j > my - mbc);
    if (!band) return;
    const int p = patches[pi];
    const double alpha = la.a[desc[p].level & 31];
    const size_t base = (size_t)p * nxy * meqn;
    for (int m = 0; m < meqn; m++) {
        const size_t k = base + (size_t)m * nxy + c;
        qi[k] = ql[k] + alpha * (q[k] - ql[k]);
    }
}
__global__ void k_timeinterp(const double* __restrict__ q, const double* __restrict__ ql, double* __restrict__ qi,
                             const int* __restrict__ patches, int npatch, const PatchDesc* __restrict__ desc, int mx,
                             int my, int mbc, int meqn, LevelAlpha la)
{
    grid_dependency_wait();       // programmatic launch: the previous grid's writes are visible
    grid_launch_dependents();
    const long t = flat_index();
    if (t < (long)npatch * (mx + 2 * mbc) * (my + 2 * mbc))
        timeinterp_at(q, ql, qi, patches, desc, mx, my, mbc, meqn, la, t);
}

// ---------------------------------------------------------------------------
// Time sync
// ---------------------------------------------------------------------------
struct RegOff {
    int fp0, fp1, fm0, fm1, gp0, gp1, gm0, gm1, ef0, ef1, ef2, ef3;
    __device__ RegOff(int mx, int my, int meqn)
    {
        fp0 = 0; fp1 = my * meqn; fm0 = 2 * my * meqn; fm1 = 3 * my * meqn;
        gp0 = 4 * my * meqn; gp1 = gp0 + mx * meqn; gm0 = gp0 + 2 * mx * meqn; gm1 = gp0 + 3 * mx * meqn;
        ef0 = gp0 + 4 * mx * meqn; ef1 = ef0 + 2 * my * meqn; ef2 = ef1 + 2 * my * meqn; ef3 = ef2 + 2 * mx * meqn;
    }
};

// The corrections of a time sync, one CTA per patch of the synced levels.  A face of a
// patch is either same-size (one samesize op) or half-size (two f2c ops,
// igrid 0 and 1, each covering half the face), so every (face, tangential index,
// field) has at most one correction.  The CTA files the patch's ops by face in
// shared memory, computes every correction with one thread each (phase 1), then
// adds them to the boundary cells with one thread per (cell, field) (phase 2):
// a corner cell on two corrected faces takes the samesize corrections first,
// then the f2c ones, each kind in face order -- the order of the reference's
// additions to that cell.  Every op reads registers only, which no correction
// writes.
//   samesize: clawpack46_fort_time_sync_samesize (same orientation, sc = 1),
//             clawpack46_time_sync.f:528-704: delta = (ef_n - ef_t) - (f_n - f_t),
//             q += 0.5 delta / area
//   f2c:      clawpack46_fort_time_sync_f2c (same orientation, sc = 1),
//             clawpack46_time_sync.f:254-498: the fine pair d, d+1 (d = 1 + n_off + 2 j)
//             of coarse cell j, skipped when outside the fine face; q += deltac / area
// Scratch: the ops below and 4 * meqn * max(mx, my) doubles (corrections) followed
// by as many flag bytes (sync_scratch_bytes), then the prefetched registers and cells
// (sync_prefetch_bytes), in dynamic shared memory.
struct SyncSmem { SyncOp op[8]; int ss[4]; int fc[4][2]; };   // op slots per face (-1: none)
__host__ __device__ constexpr size_t sync_scratch_bytes(int mx, int my, int meqn)
{
    return ((size_t)4 * meqn * (mx > my ? mx : my) * (sizeof(double) + 1) + 15) / 16 * 16;
}
__host__ __device__ constexpr size_t sync_prefetch_bytes(int mx, int my, int meqn)
{
    return ((size_t)2 * 4 * meqn * (mx > my ? mx : my) + (size_t)(2 * (mx + my) - 4) * meqn) * sizeof(double);
}
// 8-byte asynchronous copy global -> shared (cp.async, sm_80+), and the wait for this
// thread's copies
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Patch shape and field count of the time sync: compile-time for the common shapes
// (the index arithmetic and register offsets fold), run-time otherwise.
template <int MX, int MEQN>
struct FixedSync {
    static constexpr int mx = MX, my = MX, mbc = 2, meqn = MEQN;
    __device__ FixedSync(int, int, int, int) {}
};
struct RunSync {
    int mx, my, mbc, meqn;
    __device__ RunSync(int mx_, int my_, int mbc_, int meqn_) : mx(mx_), my(my_), mbc(mbc_), meqn(meqn_) {}
};
template <class PS>
__device__ void sync_group(const PS& P, int p, int tid, int nthr, SyncSmem& S, double* s_corr,
                           double* __restrict__ q, const double* __restrict__ regs,
                           const PatchDesc* __restrict__ desc, const SyncOp* __restrict__ ops, int nreg)
{
    const int mx = P.mx, my = P.my, mbc = P.mbc, meqn = P.meqn;
    const int nmax = mx > my ? mx : my;
    unsigned char* s_has = reinterpret_cast<unsigned char*>(s_corr + 4 * meqn * nmax);
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc, nxy = nx * ny;
    const int n1 = 4 * meqn * nmax;                            // phase-1 items: (face, field, index)
    const int ring = 2 * (mx + my) - 4;                        // interior cells on the patch boundary
    const int n2 = ring * meqn;                                // phase-2 items: (cell, field)
    RegOff R(mx, my, meqn);
    const double* rt = regs + (size_t)p * nreg;
    // phase-1 item t: face, field, index, its length, and this patch's two registers the
    // correction reads (A: edge flux, B: fluctuation sum) at the face's side
    auto item1 = [&](int t, int& face, int& m, int& j, int& nt, int& ra, int& rb) {
        face = t / (meqn * nmax);
        const int r = t % (meqn * nmax);
        m = r / nmax;
        j = r % nmax;
        nt = (face < 2) ? my : mx;
        const int o = j + m * nt;
        ra = (face == 0 ? R.ef0 : face == 1 ? R.ef1 : face == 2 ? R.ef2 : R.ef3) + o;
        rb = (face == 0 ? R.fp0 : face == 1 ? R.fm1 : face == 2 ? R.gp0 : R.gm1) + o;
    };
    // phase-2 item t: the cell's offset in q (field m plane) and its x and y faces
    auto item2 = [&](int t, int& m, int& ic, int& jc) {
        m = t / ring;
        const int k = t % ring;
        if (k < mx) { ic = mbc + k; jc = mbc; }
        else if (k < 2 * mx) { ic = mbc + k - mx; jc = my + mbc - 1; }
        else if (k < 2 * mx + my - 2) { ic = mbc; jc = mbc + 1 + (k - 2 * mx); }
        else { ic = mx + mbc - 1; jc = mbc + 1 + (k - 2 * mx - (my - 2)); }
    };
    double* qp = q + (size_t)p * nxy * meqn;
    // this patch's registers of every phase-1 item and boundary cells of every phase-2
    // item, copied into shared memory (asynchronously, no registers held) while the
    // ops arrive: neither depends on them.  Each thread reads back only its own items.
    double* pre_r = s_corr + sync_scratch_bytes(mx, my, meqn) / sizeof(double);   // [n1][2]
    double* pre_q = pre_r + 2 * n1;                                                // [n2]
    for (int t = tid; t < n1; t += nthr) {
        int face, m, j, nt, ra, rb;
        item1(t, face, m, j, nt, ra, rb);
        if (j < nt) { cp_async8(pre_r + 2 * t, rt + ra); cp_async8(pre_r + 2 * t + 1, rt + rb); }
    }
    for (int t = tid; t < n2; t += nthr) {
        int m, ic, jc;
        item2(t, m, ic, jc);
        cp_async8(pre_q + t, qp + (size_t)m * nxy + jc * nx + ic);
    }
    const double area = desc[p].dx * desc[p].dy;
    if (tid < 4) { S.ss[tid] = -1; S.fc[tid][0] = -1; S.fc[tid][1] = -1; }
    if (tid < SYNC_SLOTS) S.op[tid] = ops[(size_t)p * SYNC_SLOTS + tid];
    __syncthreads();
    if (S.op[0].kind == SYNC_NONE) {                           // no corrections for this patch
        cp_async_wait_all();
        return;
    }
    if (tid < SYNC_SLOTS) {
        const SyncOp& op = S.op[tid];
        if (op.kind == SYNC_SAMESIZE) S.ss[op.face & 3] = tid;
        else if (op.kind == SYNC_F2C) S.fc[op.face & 3][op.igrid & 1] = tid;
    }
    __syncthreads();
    cp_async_wait_all();
    // ---- phase 1: the correction of each (face, field, tangential index) ----
    for (int t = tid; t < n1; t += nthr) {
        int face, m, j, nt, ra, rb;
        item1(t, face, m, j, nt, ra, rb);
        bool has = false;
        double corr = 0.0;
        if (j < nt) {
            const double rA = pre_r[2 * t], rB = pre_r[2 * t + 1];
            if (S.ss[face] >= 0) {
                const SyncOp& op = S.op[S.ss[face]];
                const double* rn = regs + (size_t)op.n * nreg;
                double delta;
                if (face == 0) {
                    double fp = rn[R.fp1 + j + m * my];
                    double ef = 1 * rn[R.ef1 + j + m * my + my * meqn];
                    delta = (ef - rA) - (fp - rB);
                } else if (face == 1) {
                    double fm = rn[R.fm0 + j + m * my];
                    double ef = 1 * rn[R.ef0 + j + m * my + my * meqn];
                    delta = (rA - ef) - (fm - rB);
                } else if (face == 2) {
                    double gp = rn[R.gp1 + j + m * mx];
                    double ef = 1 * rn[R.ef3 + j + m * mx + mx * meqn];
                    delta = (ef - rA) - (gp - rB);
                } else {
                    double gm = rn[R.gm0 + j + m * mx];
                    double ef = 1 * rn[R.ef2 + j + m * mx + mx * meqn];
                    delta = (rA - ef) - (gm - rB);
                }
                corr = 0.5 * delta / area;
                has = true;
            } else {
                for (int ig = 0; ig < 2 && !has; ig++) {
                    if (S.fc[face][ig] < 0) continue;
                    const SyncOp& op = S.op[S.fc[face][ig]];
                    const int d = 1 + op.n_off + 2 * j;        // first fine child (Fortran index)
                    if (d < 1 || d + 1 > nt) continue;         // fc46_skip_this_grid
                    const double* rn = regs + (size_t)op.n * nreg;
                    const int f0 = d - 1, f1 = d;              // 0-based fine pair
                    double deltac;
                    if (face == 0) {
                        double fp = rn[R.fp1 + f0 + m * my] + rn[R.fp1 + f1 + m * my];
                        double ef = 1 * (rn[R.ef1 + f0 + m * my + my * meqn] + rn[R.ef1 + f1 + m * my + my * meqn]);
                        deltac = (ef - rA) - (fp - rB);
                    } else if (face == 1) {
                        double fm = rn[R.fm0 + f0 + m * my] + rn[R.fm0 + f1 + m * my];
                        double ef = 1 * (rn[R.ef0 + f0 + m * my + my * meqn] + rn[R.ef0 + f1 + m * my + my * meqn]);
                        deltac = (rA - ef) - (fm - rB);
                    } else if (face == 2) {
                        double gp = rn[R.gp1 + f0 + m * mx] + rn[R.gp1 + f1 + m * mx];
                        double ef = 1 * (rn[R.ef3 + f0 + m * mx + mx * meqn] + rn[R.ef3 + f1 + m * mx + mx * meqn]);
                        deltac = (ef - rA) - (gp - rB);
                    } else {
                        double gm = rn[R.gm0 + f0 + m * mx] + rn[R.gm0 + f1 + m * mx];
                        double ef = 1 * (rn[R.ef2 + f0 + m * mx + mx * meqn] + rn[R.ef2 + f1 + m * mx + mx * meqn]);
                        deltac = (rA - ef) - (gm - rB);
                    }
                    corr = deltac / area;
                    has = true;
                }
            }
        }
        s_corr[t] = corr;
        s_has[t] = has ? 1 : 0;
    }
    __syncthreads();
    // ---- phase 2: add them to the boundary cells, samesize faces first ----
    for (int t = tid; t < n2; t += nthr) {
        int m, ic, jc;                                         // storage indices of the cell
        item2(t, m, ic, jc);
        const int fx = (ic == mbc) ? 0 : (ic == mx + mbc - 1) ? 1 : -1;
        const int fy = (jc == mbc) ? 2 : (jc == my + mbc - 1) ? 3 : -1;
        // slots of the cell's corrections on its x and y faces, in the reference's order
        int sl[2] = {-1, -1};
        if (fx >= 0) sl[0] = (fx * meqn + m) * nmax + (jc - mbc);
        if (fy >= 0) sl[1] = (fy * meqn + m) * nmax + (ic - mbc);
        const bool xss = fx >= 0 && S.ss[fx] >= 0, yss = fy >= 0 && S.ss[fy] >= 0;
        const int first = (!xss && yss) ? 1 : 0;               // a samesize y face goes before an f2c x face
        double* qq = qp + (size_t)m * nxy + jc * nx + ic;
        double v = 0.0;
        bool touched = false;
        for (int w = 0; w < 2; w++) {
            const int s = sl[w ^ first];
            if (s < 0 || !s_has[s]) continue;
            if (!touched) { v = pre_q[t]; touched = true; }
            v = v + s_corr[s];
        }
        if (touched) *qq = v;
    }
}
// One CTA per patch of the synced levels: 128 threads and at most 32 registers, 16
// CTAs per SM, so a sync of up to ~2300 patches runs in one wave.
template <class PS>
__global__ void __launch_bounds__(128, 16)
k_sync(double* __restrict__ q, const double* __restrict__ regs, const PatchDesc* __restrict__ desc,
       const SyncOp* __restrict__ ops, int p0, int mx, int my, int mbc, int meqn, int nreg)
{
    grid_dependency_wait();       // programmatic launch: the previous grid's writes are visible
    grid_launch_dependents();
    __shared__ SyncSmem S;
    extern __shared__ double s_corr[];
    sync_group(PS(mx, my, mbc, meqn), p0 + blockIdx.x, threadIdx.x, blockDim.x, S, s_corr, q, regs, desc, ops, nreg);
}

// fclaw2d_time_sync's resets for levels [minlevel, maxl] (src/fclaw2d_time_sync.c:118-154):
// same-size faces of every synced level, coarse/fine faces of each synced pair
// (half-size faces of levels < maxl, double-size faces of levels > minlevel) and
// physical faces.  One index per (patch, face, register entry of that face).
__device__ __forceinline__ long reset_sync_items(int np, int mx, int my, int meqn)
{
    return (long)np * 4 * meqn * (mx > my ? mx : my);
}
__device__ __forceinline__ void reset_sync_at(double* __restrict__ regs, const PatchDesc* __restrict__ desc, int p0,
                                              int mx, int my, int meqn, int nreg, int minlevel, int maxl, long t)
{
    const int per = meqn * (mx > my ? mx : my);
    const int pi = (int)(t / (4 * per)), r = (int)(t - (long)pi * 4 * per), k = r / per, u = r - k * per;
    if (u >= meqn * (k < 2 ? my : mx)) return;
    const int p = p0 + pi;
    const PatchDesc& pd = desc[p];
    const int L = pd.level;
    const int ft = (pd.face_type >> (2 * k)) & 3;            // 0 bnd, 1 half, 2 same, 3 double
    bool reset;
    if (ft == 2) reset = true;
    else if (ft == 1) reset = L < maxl;
    else if (ft == 3) reset = L - 1 >= minlevel && L - 1 < maxl;
    else reset = true;
    if (!reset) return;
    double* r0 = regs + (size_t)p * nreg;
    RegOff R(mx, my, meqn);
    if (k < 2) {
        r0[(k == 0 ? R.fm0 : R.fm1) + u] = 0.0;
        r0[(k == 0 ? R.fp0 : R.fp1) + u] = 0.0;
        const int ef = (k == 0) ? R.ef0 : R.ef1;
        r0[ef + u] = 0.0;
        r0[ef + u + meqn * my] = 0.0;
    } else {
        r0[(k == 2 ? R.gm0 : R.gm1) + u] = 0.0;
        r0[(k == 2 ? R.gp0 : R.gp1) + u] = 0.0;
        const int ef = (k == 2) ? R.ef2 : R.ef3;
        r0[ef + u] = 0.0;
        r0[ef + u + meqn * mx] = 0.0;
    }
}
__global__ void k_reset_sync(double* __restrict__ regs, const PatchDesc* __restrict__ desc, int p0, int np, int mx,
                             int my, int meqn, int nreg, int minlevel, int maxl)
{
    grid_dependency_wait();       // programmatic launch: the previous grid's writes are visible
    grid_launch_dependents();
    const long t = flat_index();
    if (t < reset_sync_items(np, mx, my, meqn)) reset_sync_at(regs, desc, p0, mx, my, meqn, nreg, minlevel, maxl, t);
}

// Per-patch, per-field Kahan sums of q*dx*dy over interior cells in (j, i) order.
__global__ void k_patch_mass(const double* __restrict__ q, const PatchDesc* __restrict__ desc, int mx, int my,
                             int mbc, int meqn, double* __restrict__ out, const double* __restrict__ areas)
{
    const int p = blockIdx.x, m = threadIdx.x;
    if (m >= meqn) return;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const PatchDesc pd = desc[p];
    const double area = pd.dx * pd.dy;
    const double* qp = q + ((size_t)p * meqn + m) * nx * ny;
    // manifold: the cell areas (area(i,j), fclaw2d_clawpatch46_diagnostics.f:40-42)
    const double* ap = areas ? areas + (size_t)p * (nx + 2) * (ny + 2) : nullptr;
    double sum = 0.0, comp = 0.0;
    for (int j = 0; j < my; j++)
        for (int i = 0; i < mx; i++) {
            const double aij = ap ? ap[(j + mbc + 1) * (nx + 2) + i + mbc + 1] : area;
            double y = qp[(j + mbc) * nx + i + mbc] * aij - comp;
            double t = sum + y;
            comp = (t - sum) - y;
            sum = t;
        }
    out[(size_t)p * meqn + m] = sum;
}

// Tagging tests of one patch (fort_4.6/fclaw2d_clawpatch46_tag4refinement.f:11-75 and the
// per-patch part of _tag4coarsening.f:80-130) with the criteria of
// fort_user/fclaw2d_clawpatch_*_exceeds_th.f90 on field mq (0-based plane):
//   value:      q over the padded patch exceeds the threshold;
//   difference: max(|q(i+1,j)-q(i-1,j)|, |q(i,j+1)-q(i,j-1)|) over interior cells;
//   gradient:   sqrt(dqx^2 + dqy^2 + 0^2) of central differences over interior cells
//               (times dx for TAG_GRADIENT_DX);
//   minmax:     range of q over the padded patch (the family test combines the ranges).
// Only whether some cell exceeds matters, so the reference's running minimum and
// maximum reduce to the patch's.
__global__ void k_tag(const double* __restrict__ q, const PatchDesc* __restrict__ desc, int mx, int my, int mbc,
                      int meqn, int crit, int mq, double rthr, double cthr, int* __restrict__ flags,
                      double* __restrict__ minmax)
{
    const int p = blockIdx.x;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const PatchDesc pd = desc[p];
    const double* qp = q + (size_t)p * meqn * nx * ny + (size_t)mq * nx * ny;
    if (crit == FC2D_B200_TAG_MINMAX) {
        __shared__ double smn[128], smx[128];
        double mn = qp[mbc * nx + mbc], mxv = mn;
        for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
            mn = fmin(mn, qp[c]);
            mxv = fmax(mxv, qp[c]);
        }
        smn[threadIdx.x] = mn; smx[threadIdx.x] = mxv;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) {
                smn[threadIdx.x] = fmin(smn[threadIdx.x], smn[threadIdx.x + w]);
                smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + w]);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            minmax[2 * p] = smn[0];
            minmax[2 * p + 1] = smx[0];
            flags[p] = (smx[0] - smn[0] > rthr) ? 1 : 0;
        }
        return;
    }
    int refine = 0, exceed_c = 0;
    if (crit == FC2D_B200_TAG_VALUE) {
        for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
            refine |= (qp[c] > rthr);
            exceed_c |= (qp[c] > cthr);
        }
    } else {
        const double dx2 = 2 * pd.dx, dy2 = 2 * pd.dy;
        for (int c = threadIdx.x; c < mx * my; c += blockDim.x) {
            const int i = c % mx + mbc, j = c / mx + mbc;
            double v;
            if (crit == FC2D_B200_TAG_DIFFERENCE) {
                const double dqx = fabs(qp[j * nx + i + 1] - qp[j * nx + i - 1]);
                const double dqy = fabs(qp[(j + 1) * nx + i] - qp[(j - 1) * nx + i]);
                v = fmax(dqx, dqy);
            } else {
                const double dqx = (qp[j * nx + i + 1] - qp[j * nx + i - 1]) / dx2;
                const double dqy = (qp[(j + 1) * nx + i] - qp[(j - 1) * nx + i]) / dy2;
                v = sqrt(dqx * dqx + dqy * dqy + 0.0 * 0.0);
                if (crit == FC2D_B200_TAG_GRADIENT_DX) v = v * pd.dx;
            }
            refine |= (v > rthr);
            exceed_c |= (v > cthr);
        }
    }
    refine = __syncthreads_or(refine);
    exceed_c = __syncthreads_or(exceed_c);
    if (threadIdx.x == 0) flags[p] = (refine ? 1 : 0) | (exceed_c ? 0 : 2);
}

// Halo payload of a partitioned forest: per listed patch its q, qlast and
// registers, one after another (nq + nq + nreg doubles), patch after patch.
__global__ void k_pack_patches(const int* __restrict__ slots, int n, const double* __restrict__ q,
                               const double* __restrict__ qlast, const double* __restrict__ regs, int nq, int nreg,
                               double* __restrict__ out)
{
    const int k = blockIdx.x;
    if (k >= n) return;
    const size_t per = 2 * (size_t)nq + nreg;
    const int p = slots[k];
    double* o = out + (size_t)k * per;
    for (int i = threadIdx.x; i < nq; i += blockDim.x) {
        o[i] = q[(size_t)p * nq + i];
        o[nq + i] = qlast[(size_t)p * nq + i];
    }
    for (int i = threadIdx.x; i < nreg; i += blockDim.x) o[2 * nq + i] = regs[(size_t)p * nreg + i];
}

__global__ void k_unpack_patches(const int* __restrict__ slots, int n, double* __restrict__ q,
                                 double* __restrict__ qlast, double* __restrict__ regs, int nq, int nreg,
                                 const double* __restrict__ in)
{
    const int k = blockIdx.x;
    if (k >= n) return;
    const size_t per = 2 * (size_t)nq + nreg;
    const int p = slots[k];
    const double* v = in + (size_t)k * per;
    for (int i = threadIdx.x; i < nq; i += blockDim.x) {
        q[(size_t)p * nq + i] = v[i];
        qlast[(size_t)p * nq + i] = v[nq + i];
    }
    for (int i = threadIdx.x; i < nreg; i += blockDim.x) regs[(size_t)p * nreg + i] = v[2 * nq + i];
}

// Regrid repopulation (cb_fclaw2d_regrid_repopulate, fclaw2d_regrid.c:93-205).
__global__ void k_repop(const RepopOp* __restrict__ ops, int mx, int my, int mbc, int meqn, int nreg,
                        const double* __restrict__ oq, double* __restrict__ nq,
                        const double* __restrict__ oql, double* __restrict__ nql,
                        const double* __restrict__ oqi, double* __restrict__ nqi,
                        const double* __restrict__ oregs, double* __restrict__ nregs,
                        const double* __restrict__ oarea, const double* __restrict__ narea)
{
    const RepopOp op = ops[blockIdx.x];
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc, nxy = nx * ny, nqp = nxy * meqn;
    const int ax = nx + 2, na = ax * (ny + 2);
    // area of Fortran cell (i, j) of a manifold patch's area array
    auto aidx = [&](int i, int j) { return (j + mbc) * ax + (i + mbc); };
    double* d = nq + (size_t)op.dst * nqp;
    if (op.kind == 0) {
        const size_t so = (size_t)op.src * nqp;
        for (int k = threadIdx.x; k < nqp; k += blockDim.x) {
            d[k] = oq[so + k];
            nql[(size_t)op.dst * nqp + k] = oql[so + k];
            if (nqi) nqi[(size_t)op.dst * nqp + k] = oqi[so + k];
        }
        for (int k = threadIdx.x; k < nreg; k += blockDim.x)
            nregs[(size_t)op.dst * nreg + k] = oregs[(size_t)op.src * nreg + k];
        return;
    }
    // new patch: zero everything first
    for (int k = threadIdx.x; k < nqp; k += blockDim.x) {
        d[k] = 0.0;
        nql[(size_t)op.dst * nqp + k] = 0.0;
        if (nqi) nqi[(size_t)op.dst * nqp + k] = 0.0;
    }
    for (int k = threadIdx.x; k < nreg; k += blockDim.x) nregs[(size_t)op.dst * nreg + k] = 0.0;
    __syncthreads();
    if (op.kind == 1) {
        // interpolate2fine (interpolate.f:324-392)
        const double* qc = oq + (size_t)op.src * nqp;
        const int ig = op.igrid % 2, jg = op.igrid / 2;
        const int i1 = 1 - ig, i2 = mx / 2 + (1 - ig), j1 = 1 - jg, j2 = my / 2 + (1 - jg);
        const int icadd = ig * mx / 2, jcadd = jg * my / 2;
        const int ni = i2 - i1 + 1, nj = j2 - j1 + 1;
        for (int t = threadIdx.x; t < ni * nj * meqn; t += blockDim.x) {
            const int i = i1 + t % ni, j = j1 + (t / ni) % nj, m = t / (ni * nj);
            const int ic = i + icadd, jc = j + jcadd;
            const double* c0 = qc + (size_t)m * nxy + (jc + mbc - 1) * nx + (ic + mbc - 1);
            double q0 = c0[0];
            double sl = (q0 - c0[-1]);
            double sr = (c0[1] - q0);
            double gradx = compute_slopes(sl, sr);
            sl = (q0 - c0[-nx]);
            sr = (c0[nx] - q0);
            double grady = compute_slopes(sl, sr);
            double v[2][2];
            for (int ii = 1; ii <= 2; ii++)
                for (int jj = 1; jj <= 2; jj++) {
                    const double shx = (ii - 2 / 2.0 - 0.5) / 2, shy = (jj - 2 / 2.0 - 0.5) / 2;
                    v[ii - 1][jj - 1] = q0 + shx * gradx + shy * grady;
                }
            if (narea && i >= 1 && i <= mx / 2 && j >= 1 && j <= my / 2) {
                // fclaw2d_clawpatch46_fort_fixcapaq2 (interpolate.f:409-470): the four
                // fine cells get the coarse cell's mass back, (qc kc - sum kf qf) / 4 each
                const double* af = narea + (size_t)op.dst * na;
                double sum = 0.0;
                for (int ii = 1; ii <= 2; ii++)
                    for (int jj = 1; jj <= 2; jj++)
                        sum = sum + af[aidx((i - 1) * 2 + ii, (j - 1) * 2 + jj)] * v[ii - 1][jj - 1];
                const double kc = oarea[(size_t)op.src * na + aidx(ic, jc)];
                const double cons_diff = (q0 * kc - sum) / 4.0;
                for (int ii = 1; ii <= 2; ii++)
                    for (int jj = 1; jj <= 2; jj++)
                        v[ii - 1][jj - 1] = v[ii - 1][jj - 1] + cons_diff / af[aidx((i - 1) * 2 + ii, (j - 1) * 2 + jj)];
            }
            for (int ii = 1; ii <= 2; ii++)
                for (int jj = 1; jj <= 2; jj++) {
                    const int fi = (i - 1) * 2 + ii, fj = (j - 1) * 2 + jj;
                    d[(size_t)m * nxy + (fj + mbc - 1) * nx + (fi + mbc - 1)] = v[ii - 1][jj - 1];
                }
        }
    } else {
        // average2coarse (average.f:282-364): child c fills quarter (ig, jg)
        for (int c = 0; c < 4; c++) {
            const double* qf = oq + (size_t)op.child[c] * nqp;
            const int ig = c % 2, jg = c / 2;
            const int icadd = ig * mx / 2, jcadd = jg * mx / 2;
            for (int t = threadIdx.x; t < (mx / 2) * (my / 2) * meqn; t += blockDim.x) {
                const int i = 1 + t % (mx / 2), j = 1 + (t / (mx / 2)) % (my / 2), m = t / ((mx / 2) * (my / 2));
                double sum = 0.0;
                if (narea) {
                    // manifold (average.f:340-352): sum(kf qf) / kc with the new coarse areas
                    const double* af = oarea + (size_t)op.child[c] * na;
                    for (int jj = 1; jj <= 2; jj++)
                        for (int ii = 1; ii <= 2; ii++) {
                            const int fi = (i - 1) * 2 + ii, fj = (j - 1) * 2 + jj;
                            sum = sum + af[aidx(fi, fj)] * qf[(size_t)m * nxy + (fj + mbc - 1) * nx + (fi + mbc - 1)];
                        }
                    const double kc = narea[(size_t)op.dst * na + aidx(i + icadd, j + jcadd)];
                    d[(size_t)m * nxy + (j + jcadd + mbc - 1) * nx + (i + icadd + mbc - 1)] = sum / kc;
                    continue;
                }
                for (int jj = 1; jj <= 2; jj++)
                    for (int ii = 1; ii <= 2; ii++) {
                        const int fi = (i - 1) * 2 + ii, fj = (j - 1) * 2 + jj;
                        sum = sum + qf[(size_t)m * nxy + (fj + mbc - 1) * nx + (fi + mbc - 1)];
                    }
                d[(size_t)m * nxy + (j + jcadd + mbc - 1) * nx + (i + icadd + mbc - 1)] = sum / 4;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
// Whole-patch copies src -> dst of the listed slots (restores ghost cells).
__global__ void k_restore_patches(double* __restrict__ dst, const double* __restrict__ src, const int* __restrict__ slots,
                                  int nq)
{
    const size_t base = (size_t)slots[blockIdx.x] * nq;
    for (int k = threadIdx.x; k < nq; k += blockDim.x) dst[base + k] = src[base + k];
}
void launch_restore_patches(const Dims& d, double* dst, const double* src, const int* slots, int n, cudaStream_t st)
{
    if (n > 0) k_restore_patches<<<n, 256, 0, st>>>(dst, src, slots, d.nq());
}

void launch_average_copy(const Dims& d, const GatherSeg<FillOp>& a0, const GatherSeg<FillOp>& a1,
                         const GatherSeg<FillOp>& c0, const GatherSeg<FillOp>& c1, const double* area,
                         cudaStream_t st)
{
    const long n = ((long)a0.n + a1.n + c0.n + c1.n) * d.mbc * (d.mx > d.my ? d.mx : d.my);
    if (n <= 0) return;
    auto kern = area ? &k_average_copy<RunShape, true> : &k_average_copy<RunShape, false>;
    if (!area && d.mx == d.my && d.mbc == 2) {
        if (d.mx == 8) kern = &k_average_copy<FixedShape<8, 2>, false>;
        else if (d.mx == 16) kern = &k_average_copy<FixedShape<16, 2>, false>;
        else if (d.mx == 32) kern = &k_average_copy<FixedShape<32, 2>, false>;
    }
    launch_k(kern, nblk(n, 256), 256, 0, st, a0, a1, c0, c1, d.mx, d.my, d.mbc, d.meqn, area);
}
void launch_interp(const Dims& d, const GatherSeg<InterpEnt>& s0, const GatherSeg<InterpEnt>& s1, cudaStream_t st)
{
    const long n = ((long)s0.n + s1.n) * d.meqn;
    if (n > 0) launch_k(k_interp, nblk(n, 256), 256, 0, st, s0, s1, d.nx(), d.nxy(), d.meqn);
}
void launch_phys(const Dims& d, const GatherSeg<PhysEnt>& s0, const GatherSeg<PhysEnt>& s1, const double* bcstate,
                 cudaStream_t st)
{
    const long n = ((long)s0.n + s1.n) * d.meqn;
    if (n > 0) launch_k(k_phys, nblk(n, 256), 256, 0, st, s0, s1, d.nxy(), d.meqn, bcstate);
}
void launch_timeinterp(const Dims& d, const double* q, const double* qlast, double* qinterp, const int* patches,
                       int npatch, const PatchDesc* desc, const LevelAlpha& alpha, cudaStream_t st)
{
    if (npatch > 0)
        launch_k(k_timeinterp, nblk((long)npatch * d.nxy(), 256), 256, 0, st, q, qlast, qinterp, patches, npatch, desc,
                 d.mx, d.my, d.mbc, d.meqn, alpha);
}
void launch_sync(const Dims& d, double* q, const double* regs, const PatchDesc* desc, const SyncOp* ops, int p0,
                 int np, cudaStream_t st)
{
    if (np <= 0) return;
    auto kern = &k_sync<RunSync>;
    if (d.mx == d.my && d.mbc == 2) {
        if (d.mx == 16 && d.meqn == 3) kern = &k_sync<FixedSync<16, 3>>;
        else if (d.mx == 16 && d.meqn == 4) kern = &k_sync<FixedSync<16, 4>>;
        else if (d.mx == 8 && d.meqn == 3) kern = &k_sync<FixedSync<8, 3>>;
    }
    launch_k(kern, np, 128, sync_scratch_bytes(d.mx, d.my, d.meqn) + sync_prefetch_bytes(d.mx, d.my, d.meqn), st, q,
             regs, desc, ops, p0, d.mx, d.my, d.mbc, d.meqn, d.nreg());
}
void launch_reset_sync(const Dims& d, double* regs, const PatchDesc* desc, int p0, int np, int minlevel, int maxl,
                       cudaStream_t st)
{
    const long n = (long)np * 4 * d.meqn * (d.mx > d.my ? d.mx : d.my);
    if (np > 0)
        launch_k(k_reset_sync, nblk(n, 256), 256, 0, st, regs, desc, p0, np, d.mx, d.my, d.meqn, d.nreg(), minlevel,
                 maxl);
}
void launch_patch_mass(const Dims& d, const double* q, const PatchDesc* desc, int np, double* out, cudaStream_t st,
                       const double* area)
{
    if (np > 0) k_patch_mass<<<np, 32, 0, st>>>(q, desc, d.mx, d.my, d.mbc, d.meqn, out, area);
}
void launch_tag(const Dims& d, const double* q, const PatchDesc* desc, int np, int crit, int mq, double rthr,
                double cthr, int* flags, cudaStream_t st, double* minmax)
{
    if (np > 0) k_tag<<<np, 128, 0, st>>>(q, desc, d.mx, d.my, d.mbc, d.meqn, crit, mq, rthr, cthr, flags, minmax);
}
void launch_pack_patches(const Dims& d, const int* slots, int n, const double* q, const double* qlast,
                         const double* regs, double* out, cudaStream_t st)
{
    if (n > 0) k_pack_patches<<<n, 256, 0, st>>>(slots, n, q, qlast, regs, d.nq(), d.nreg(), out);
}
void launch_unpack_patches(const Dims& d, const int* slots, int n, double* q, double* qlast, double* regs,
                           const double* in, cudaStream_t st)
{
    if (n > 0) k_unpack_patches<<<n, 256, 0, st>>>(slots, n, q, qlast, regs, d.nq(), d.nreg(), in);
}
// aux of a new forest, one CTA per new slot: src >= 0 the old slot's, src <= -2 staged
// patch -2 - src, src = -1 left to the cubed-sphere metric
__global__ void k_aux_repop(const int* __restrict__ src, int naux, const double* __restrict__ oaux,
                            const double* __restrict__ staged, double* __restrict__ aux)
{
    const int i = blockIdx.x, sidx = src[i];
    if (sidx == -1) return;
    const double* from = sidx >= 0 ? oaux + (size_t)sidx * naux : staged + (size_t)(-2 - sidx) * naux;
    double* to = aux + (size_t)i * naux;
    for (int k = threadIdx.x; k < naux; k += blockDim.x) to[k] = from[k];
}
void launch_aux_repop(const Dims& d, const int* src, int n, const double* oaux, const double* staged, double* aux,
                      cudaStream_t st)
{
    if (n > 0 && d.maux > 0) k_aux_repop<<<n, 256, 0, st>>>(src, d.naux(), oaux, staged, aux);
}

void launch_repop(const Dims& d, const RepopOp* ops, int nops, const double* oq, double* nq, const double* oqlast,
                  double* nqlast, const double* oqi, double* nqi, const double* oregs, double* nregs,
                  const double* oarea, const double* narea, cudaStream_t st)
{
    if (nops > 0)
        k_repop<<<nops, 256, 0, st>>>(ops, d.mx, d.my, d.mbc, d.meqn, d.nreg(), oq, nq, oqlast, nqlast, oqi, nqi,
                                      oregs, nregs, oarea, narea);
}

}  // namespace fcb
