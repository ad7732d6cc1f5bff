// host_forest.cpp -- forest, neighbour relations, adaptation and gather tables.
//
// Neighbour semantics restate p4est's on a 2:1 face+corner balanced forest as
// ForestClaw consumes them (src/fclaw2d_regrid.c:337-400, src/fclaw2d_patch.c:980-1034,
// src/fclaw2d_corner_neighbors.c:80-300).  The gather tables replay, index by
// index, the reference's ghost-fill callbacks
//   copy2ghost / average2ghost / interpolate2ghost / setphysical  (src/fclaw2d_ghost_fill.c:140-295)
//   cb_face_fill / cb_corner_fill                                  (src/fclaw2d_face_neighbors.c:195-450,
//                                                                   src/fclaw2d_corner_neighbors.c:301-535)
//   fort_4.6 copy / average / interpolate, clawpack46_bc2_default.f
// with the same-orientation transforms of src/forestclaw2d.c:609-1360 (a shift
// in brick-global cell indices, canonical child order).
#include "host_forest.hpp"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <thread>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include "fcb_sphere.h"

namespace fcb {

// ---------------------------------------------------------------------------
// cubed-sphere connectivity
// ---------------------------------------------------------------------------
// p4est's cubed connectivity (p4est_connectivity_new_cubed, called by
// fclaw2d_domain_new_cubedsphere, src/fclaw2d_convenience.c:355) is not in the
// reference tree (p4est is an empty submodule).  The same information follows
// from the mapping the reference pairs with it: two block faces are joined where
// their mapped edges coincide, with the edge parameter running the same way
// (flip 0) or reversed (flip 1).
namespace {
struct CSTable {
    CSFace f[6][4];
    CSTable()
    {
        auto edge = [](int face, double t, double& x, double& y) {
            if (face == 0) { x = 0.0; y = t; } else if (face == 1) { x = 1.0; y = t; }
            else if (face == 2) { x = t; y = 0.0; } else { x = t; y = 1.0; }
        };
        auto pt = [&](int b, int face, double t, double* p) {
            double x, y;
            edge(face, t, x, y);
            cs_map(b, x, y, &p[0], &p[1], &p[2]);
        };
        auto close = [](const double* a, const double* b) {
            return std::fabs(a[0] - b[0]) + std::fabs(a[1] - b[1]) + std::fabs(a[2] - b[2]) < 1e-9;
        };
        for (int b = 0; b < 6; b++)
            for (int fc = 0; fc < 4; fc++) {
                double p0[3], p1[3];
                pt(b, fc, 0.25, p0);
                pt(b, fc, 0.75, p1);
                CSFace& F = f[b][fc];
                F.nb = -1;
                for (int b2 = 0; b2 < 6 && F.nb < 0; b2++)
                    for (int f2 = 0; f2 < 4; f2++) {
                        if (b2 == b) continue;
                        double q0[3], q1[3];
                        pt(b2, f2, 0.25, q0);
                        pt(b2, f2, 0.75, q1);
                        if (close(p0, q0) && close(p1, q1)) { F.nb = b2; F.nf = f2; F.flip = 0; break; }
                        if (close(p0, q1) && close(p1, q0)) { F.nb = b2; F.nf = f2; F.flip = 1; break; }
                    }
                // depth d beyond face fc and position t along it, into block nb at depth d
                // inside face nf: an isometry of the plane, so affine with integer M, c
                auto T = [&](double x, double y, double& x2, double& y2) {
                    double d, t;
                    if (fc == 0) { d = -x; t = y; } else if (fc == 1) { d = x - 1.0; t = y; }
                    else if (fc == 2) { d = -y; t = x; } else { d = y - 1.0; t = x; }
                    const double sp = F.flip ? 1.0 - t : t;
                    if (F.nf == 0) { x2 = d; y2 = sp; } else if (F.nf == 1) { x2 = 1.0 - d; y2 = sp; }
                    else if (F.nf == 2) { x2 = sp; y2 = d; } else { x2 = sp; y2 = 1.0 - d; }
                };
                double cx, cy, ax, ay, bx, by;
                T(0.0, 0.0, cx, cy);
                T(1.0, 0.0, ax, ay);
                T(0.0, 1.0, bx, by);
                F.c[0] = (int)std::lround(cx); F.c[1] = (int)std::lround(cy);
                F.M[0][0] = (int)std::lround(ax - cx); F.M[1][0] = (int)std::lround(ay - cy);
                F.M[0][1] = (int)std::lround(bx - cx); F.M[1][1] = (int)std::lround(by - cy);
            }
    }
};
const CSTable& cs_table()
{
    static const CSTable t;
    return t;
}
// Worker threads kept for the life of the process (creating and joining a dozen threads
// per call cost more than the work of a small forest).  A job is n tasks handed out by a
// shared counter; the calling thread takes tasks too and returns once all n are done, so
// a job completes even if no worker wakes (another caller's job in flight, a forked
// child without the workers).  A worker that wakes after its job is done finds the
// counter spent and never calls the job's function.
class TaskPool {
public:
    static TaskPool& get()
    {
        static TaskPool* pool = new TaskPool();             // never destroyed: its threads stay detached
        return *pool;
    }
    void run(int n, int helpers, const std::function<void(int)>& fn)
    {
        auto job = std::make_shared<Job>();
        job->fn = fn;
        job->n = n;
        job->slots = std::min(helpers, nworkers_);
        {
            std::lock_guard<std::mutex> g(mu_);
            cur_ = job;
            gen_++;
        }
        cv_.notify_all();
        work(*job);
        for (int k = 0; k < SPIN && job->done.load(std::memory_order_acquire) != n; k++) std::this_thread::yield();
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return job->done.load() == n; });
    }

private:
    struct Job {
        std::function<void(int)> fn;
        int n = 0;
        std::atomic<int> next{0}, done{0}, slots{0};
    };
    TaskPool()
    {
        nworkers_ = std::max(0, std::min((int)std::thread::hardware_concurrency(), 16) - 1);
        for (int t = 0; t < nworkers_; t++) std::thread([this] { loop(); }).detach();
    }
    void work(Job& j)
    {
        for (int i; (i = j.next.fetch_add(1)) < j.n;) {
            j.fn(i);
            if (j.done.fetch_add(1) + 1 == j.n) {
                std::lock_guard<std::mutex> g(mu_);
                done_cv_.notify_all();
            }
        }
    }
    void loop()
    {
        unsigned long long seen = 0;
        for (;;) {
            std::shared_ptr<Job> job;
            // a regrid posts several jobs in a row: look for the next one for a short while
            // (bounded) before sleeping on the condition variable
            for (int k = 0; k < SPIN && gen_.load(std::memory_order_acquire) == seen; k++) std::this_thread::yield();
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_.load() != seen; });
                seen = gen_.load();
                job = cur_;
            }
            if (job->slots.fetch_sub(1) > 0) work(*job);
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::shared_ptr<Job> cur_;
    std::atomic<unsigned long long> gen_{0};
    static constexpr int SPIN = 4000;                  // yields before a worker sleeps
    int nworkers_ = 0;
};

// Runs tasks 0..n-1 on up to nt threads (the calling one included).
template <class Fn>
void run_tasks(int n, int nt, Fn fn)
{
    nt = std::max(1, std::min(nt, n));
    if (nt == 1) { for (int i = 0; i < n; i++) fn(i); return; }
    TaskPool::get().run(n, nt - 1, std::function<void(int)>(std::ref(fn)));
}

}  // namespace

const CSFace& cs_face(int b, int f) { return cs_table().f[b][f]; }

int cs_face_to(int a, int b)
{
    if (a == b) return -1;
    for (int f = 0; f < 4; f++)
        if (cs_face(a, f).nb == b) return f;
    return -1;
}

void cs_xform(int b, int f, long N, long X, long Y, long& X2, long& Y2)
{
    // cell centres (X + 1/2) / N map by the affine isometry; in integers
    // 2 X' + 1 = M (2 X + 1) + 2 N c
    const CSFace& F = cs_face(b, f);
    X2 = (F.M[0][0] * (2 * X + 1) + F.M[0][1] * (2 * Y + 1) + 2 * N * F.c[0] - 1) / 2;
    Y2 = (F.M[1][0] * (2 * X + 1) + F.M[1][1] * (2 * Y + 1) + 2 * N * F.c[1] - 1) / 2;
}

int Forest::step(int i, int l, int x, int y, int dx, int dy, int& ox, int& oy) const
{
    const Geometry& G = gi(i);
    if (G.kind == 0) {
        ox = x + dx; oy = y + dy;
        return in_domain(i, l, ox, oy) ? 1 : 0;
    }
    const long n = 1L << (l + G.lbase);
    const int b = (int)(x / n);
    const long ix = x - b * n + dx, iy = (long)y + dy;
    const bool outx = ix < 0 || ix >= n, outy = iy < 0 || iy >= n;
    if (!outx && !outy) { ox = (int)(b * n + ix); oy = (int)iy; return 1; }
    if (outx && outy) return -1;
    const int f = outx ? (ix < 0 ? 0 : 1) : (iy < 0 ? 2 : 3);
    long X2, Y2;
    cs_xform(b, f, n, ix, iy, X2, Y2);
    ox = (int)(cs_face(b, f).nb * n + X2); oy = (int)Y2;
    return 1;
}

// The bits of v at the even positions of a 64-bit word (binary magic numbers: shift and
// mask in halving steps).
static uint64_t spread_bits(uint32_t v)
{
    uint64_t x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

// Morton (Z-order) key: bit b of x at 2b, bit b of y at 2b + 1.
static uint64_t interleave(uint32_t x, uint32_t y) { return spread_bits(x) | (spread_bits(y) << 1); }

// p4est brick tree numbering: rank of the block position in Morton order.
static int brick_block(int mi, int mj, int bx, int by)
{
    uint64_t k = interleave((uint32_t)bx, (uint32_t)by);
    int r = 0;
    for (int j = 0; j < mj; j++)
        for (int i = 0; i < mi; i++)
            if (interleave((uint32_t)i, (uint32_t)j) < k) r++;
    return r;
}

// clawpatch_define geometry (fclaw2d_clawpatch.cpp:232-301, non-manifold, brick map
// fclaw2d_map_brick.c:68-77).
void Forest::geometry(PatchInfo& q) const
{
    const Geometry& g = gi(q.inst);
    const int l = q.level + g.lbase;
    const int bx = q.gx >> l, by = q.gy >> l;
    const int ix = q.gx - (bx << l), iy = q.gy - (by << l);
    const double w = 1.0 / (double)(1 << l);
    const double xl = ix * w, yl = iy * w, xu = (ix + 1) * w, yu = (iy + 1) * w;
    double xlo, ylo, xup, yup;
    if ((g.mi == 1 && g.mj == 1) || g.kind == 1) { xlo = xl; ylo = yl; xup = xu; yup = yu; }
    else {
        xlo = (double)(bx + xl) / g.mi; xup = (double)(bx + xu) / g.mi;
        ylo = (double)(by + yl) / g.mj; yup = (double)(by + yu) / g.mj;
    }
    q.block = g.kind == 1 ? bx : brick_block(g.mi, g.mj, bx, by);
    q.xlower = g.ax + (g.bx - g.ax) * xlo;
    const double xupper = g.ax + (g.bx - g.ax) * xup;
    q.ylower = g.ay + (g.by - g.ay) * ylo;
    const double yupper = g.ay + (g.by - g.ay) * yup;
    q.dx = (xupper - q.xlower) / g.d.mx;
    q.dy = (yupper - q.ylower) / g.d.my;
    const unsigned sh = (unsigned)(24 - l);
    q.morton = interleave((uint32_t)ix << sh, (uint32_t)iy << sh);
}

int Forest::lookup(int i, int l, int x, int y) const
{
    if (l < 0 || !in_domain(i, l, x, y)) return -1;
    return index_.get(key(i, l, x, y));
}

bool Forest::build(const std::vector<Leaf>& leaves, std::string& err)
{
    const int nl = (int)leaves.size();
    for (const Leaf& lf : leaves)
        if (lf.inst < 0 || lf.inst >= ninst()) { err = "leaf of an unknown instance"; return false; }
    const int nt = std::max(1, std::min((int)std::thread::hardware_concurrency(), 16));
    constexpr int CH = 256;                                     // leaves per task
    const int nch = (nl + CH - 1) / CH;
    // geometry of every leaf, and its slot key: level, instance, block, Morton
    struct SlotKey { uint64_t hi, morton; int leaf; };
    std::vector<PatchInfo>& q = scratch_;
    q.resize(nl);
    std::vector<SlotKey> ord(nl);
    run_tasks(nch, nt, [&](int c) {
        for (int i = c * CH, e = std::min(nl, i + CH); i < e; i++) {
            const Leaf& lf = leaves[i];
            PatchInfo& P = q[i];
            P = PatchInfo{};
            P.level = lf.level; P.gx = lf.gx; P.gy = lf.gy; P.inst = lf.inst;
            geometry(P);
            ord[i] = {((uint64_t)P.level << 56) | ((uint64_t)P.inst << 28) | (uint64_t)P.block, P.morton, i};
        }
    });
    std::sort(ord.begin(), ord.end(), [](const SlotKey& a, const SlotKey& b) {
        return a.hi != b.hi ? a.hi < b.hi : a.morton < b.morton;
    });
    p.resize(nl);
    run_tasks(nch, nt, [&](int c) {
        for (int i = c * CH, e = std::min(nl, i + CH); i < e; i++) p[i] = q[ord[i].leaf];
    });
    index_.reset(p.size());
    for (int i = 0; i < np(); i++) index_.put(key(p[i].inst, p[i].level, p[i].gx, p[i].gy), i);
    for (int l = 0; l < 34; l++) lev_off[l] = 0;
    minlevel_present = 99; maxlevel_present = -1;
    {
        int k = 0;
        for (int l = 0; l < 33; l++) {
            lev_off[l] = k;
            while (k < np() && p[k].level == l) k++;
            if (lev_off[l] != k) { minlevel_present = std::min(minlevel_present, l); maxlevel_present = l; }
        }
        lev_off[33] = k;
    }
    static const int FDX[4] = {-1, 1, 0, 0}, FDY[4] = {0, 0, -1, 1};
    // neighbours of every patch (independent per patch: chunks on worker threads)
    std::atomic<int> unbalanced{0};
    auto neighbours = [&](int ip) {
        PatchInfo& P = p[ip];
        const int l = P.level, in = P.inst;
        P.has_fine_nbr = 0; P.on_cf = 0;
        for (int f = 0; f < 4; f++) {
            int nx, ny;
            P.face_nbr[f][0] = P.face_nbr[f][1] = -1;
            P.phys[f] = step(in, l, P.gx, P.gy, FDX[f], FDY[f], nx, ny) != 1;
            if (P.phys[f]) { P.face_type[f] = NB_BOUNDARY; continue; }
            int k = lookup(in, l, nx, ny);
            if (k >= 0) { P.face_type[f] = NB_SAME; P.face_nbr[f][0] = k; continue; }
            k = lookup(in, l - 1, nx >> 1, ny >> 1);
            if (k >= 0) { P.face_type[f] = NB_DOUBLE; P.face_nbr[f][0] = k; P.on_cf = 1; continue; }
            // the two finer leaves across the face: our children touching it, stepped across
            int c0x, c0y, c1x, c1y;
            {
                const int ex = (f == 1) ? 1 : 0, ey = (f == 3) ? 1 : 0;
                const int kx = (f < 2) ? 0 : 1, ky = (f < 2) ? 1 : 0;
                step(in, l + 1, 2 * P.gx + ex, 2 * P.gy + ey, FDX[f], FDY[f], c0x, c0y);
                step(in, l + 1, 2 * P.gx + ex + kx, 2 * P.gy + ey + ky, FDX[f], FDY[f], c1x, c1y);
            }
            const int a = lookup(in, l + 1, c0x, c0y), b = lookup(in, l + 1, c1x, c1y);
            if (a < 0 || b < 0) { unbalanced = 1; return; }
            P.face_type[f] = NB_HALF; P.face_nbr[f][0] = a; P.face_nbr[f][1] = b;
            P.has_fine_nbr = 1; P.on_cf = 1;
        }
        for (int c = 0; c < 4; c++) {
            const int f0 = (c & 1) ? 1 : 0, f1 = (c & 2) ? 3 : 2;
            P.has_corner[c] = 0; P.corner_nbr[c] = -1; P.corner_type[c] = NB_BOUNDARY; P.bcc3[c] = 0;
            if (P.phys[f0] || P.phys[f1]) continue;            // not an interior corner
            const int ddx = (c & 1) ? 1 : -1, ddy = (c & 2) ? 1 : -1;
            int nx, ny;
            if (step(in, l, P.gx, P.gy, ddx, ddy, nx, ny) < 0) {
                // three blocks meet (src/fclaw2d_corner_neighbors.c:250-262): no corner neighbour,
                // the update's fix_corners fills these ghost cells
                P.bcc3[c] = 1;
                continue;
            }
            int k = lookup(in, l, nx, ny);
            if (k >= 0) { P.has_corner[c] = 1; P.corner_type[c] = NB_SAME; P.corner_nbr[c] = k; continue; }
            {
                int fx, fy;
                step(in, l + 1, 2 * P.gx + (ddx > 0), 2 * P.gy + (ddy > 0), ddx, ddy, fx, fy);
                k = lookup(in, l + 1, fx, fy);
            }
            if (k >= 0) {
                P.has_corner[c] = 1; P.corner_type[c] = NB_HALF; P.corner_nbr[c] = k;
                P.has_fine_nbr = 1; P.on_cf = 1; continue;
            }
            k = lookup(in, l - 1, nx >> 1, ny >> 1);
            const int cx = P.gx + (c & 1), cy = P.gy + (c >> 1);
            if (k >= 0 && (cx % 2) == 0 && (cy % 2) == 0) {   // corner point is a corner of the big leaf
                P.has_corner[c] = 1; P.corner_type[c] = NB_DOUBLE; P.corner_nbr[c] = k; P.on_cf = 1;
            }
        }
    };
    run_tasks(nch, nt, [&](int c) {
        for (int ip = c * CH, e = std::min(nl, ip + CH); ip < e; ip++) neighbours(ip);
    });
    if (unbalanced) { err = "forest is not 2:1 face balanced"; return false; }
    return true;
}

void parallel_for(int n, const std::function<void(int)>& fn) { run_tasks(n, 16, fn); }

// ---------------------------------------------------------------------------
// adaptation
// ---------------------------------------------------------------------------
// The leaves that replace patches list[0..n) of one instance (all patches: list null),
// 2:1 balanced within the instance (instances never touch one another).
static std::vector<Leaf> adapt_patches(const Forest& f, const std::vector<int>& mark, const int* list, int n,
                                       int& changed, bool threads)
{
    const int np = f.np();
    std::vector<Leaf> L;
    L.reserve(n * 2 + 8);
    std::vector<char> done(np, 0);
    changed = 0;
    for (int q = 0; q < n; q++) {
        const int i = list ? list[q] : q;
        if (done[i]) continue;
        const PatchInfo& P = f.p[i];
        if (mark[i] > 0) {
            for (int c = 0; c < 4; c++) L.push_back({P.level + 1, 2 * P.gx + (c & 1), 2 * P.gy + (c >> 1), P.inst});
            changed = 1; done[i] = 1;
        } else if (mark[i] < 0) {
            const int px = P.gx >> 1, py = P.gy >> 1, l = P.level;
            int sib[4]; bool ok = true;
            for (int c = 0; c < 4; c++) {
                sib[c] = f.lookup(P.inst, l, 2 * px + (c & 1), 2 * py + (c >> 1));
                if (sib[c] < 0 || mark[sib[c]] >= 0) ok = false;
            }
            if (ok) {
                L.push_back({l - 1, px, py, P.inst});
                for (int c = 0; c < 4; c++) done[sib[c]] = 1;
                changed = 1;
            } else {
                L.push_back({l, P.gx, P.gy, P.inst}); done[i] = 1;
            }
        } else {
            L.push_back({P.level, P.gx, P.gy, P.inst}); done[i] = 1;
        }
    }
    // 2:1 face+corner balance by refining the coarser side.  The first pass checks
    // every leaf; a later pass checks only the children the previous pass created and
    // the leaves that found a too-coarse neighbour (its children may still be too coarse).
    {
        KeyIndex idx;
        idx.reset(L.size() * 4);
        for (int i = 0; i < (int)L.size(); i++) idx.put(Forest::key(L[i].inst, L[i].level, L[i].gx, L[i].gy), i);
        std::vector<char> dead(L.size(), 0);
        std::vector<int> check(L.size());
        for (int i = 0; i < (int)L.size(); i++) check[i] = i;
        std::vector<int> ref, again;
        int kmin = 99;                                  // no leaf is coarser, now or later
        for (const Leaf& q : L) kmin = std::min(kmin, q.level);
        // leaves check[a, b): the too-coarse neighbours found (in discovery order, repeats
        // kept) and the leaves that found one
        auto scan = [&](size_t a, size_t b, std::vector<int>& found, std::vector<int>& hit) {
            for (size_t t = a; t < b; t++) {
                const int i = check[t];
                const int l = L[i].level, in = L[i].inst;
                bool any = false;
                for (int dy = -1; dy <= 1; dy++)
                    for (int dx = -1; dx <= 1; dx++) {
                        if (!dx && !dy) continue;
                        int x, y;
                        if (f.step(in, l, L[i].gx, L[i].gy, dx, dy, x, y) != 1) continue;
                        for (int k = l - 2; k >= kmin; k--) {
                            const int j = idx.get(Forest::key(in, k, x >> (l - k), y >> (l - k)));
                            if (j >= 0) { found.push_back(j); any = true; break; }
                        }
                    }
                if (any) hit.push_back(i);
            }
        };
        constexpr size_t SCAN = 512;                    // leaves per task of a threaded pass
        std::vector<std::vector<int>> found, hit;
        while (!check.empty()) {
            ref.clear();
            again.clear();
            // a pass only reads idx, so its leaves are scanned in chunks (on threads for a
            // large pass) and the chunks' findings merged in check order: the same lists
            // as one scan in order
            const size_t nc = (threads && check.size() > 2 * SCAN) ? (check.size() + SCAN - 1) / SCAN : 1;
            found.resize(std::max(found.size(), nc));
            hit.resize(std::max(hit.size(), nc));
            for (size_t c = 0; c < nc; c++) { found[c].clear(); hit[c].clear(); }
            if (nc == 1) scan(0, check.size(), found[0], hit[0]);
            else
                run_tasks((int)nc, 16, [&](int c) {
                    scan(c * SCAN, std::min(check.size(), (c + 1) * SCAN), found[c], hit[c]);
                });
            for (size_t c = 0; c < nc; c++) {
                for (int j : found[c]) if (!dead[j]) { dead[j] = 1; ref.push_back(j); }
                again.insert(again.end(), hit[c].begin(), hit[c].end());
            }
            check.clear();
            for (int i : again) if (!dead[i]) check.push_back(i);
            for (int j : ref) {
                idx.put(Forest::key(L[j].inst, L[j].level, L[j].gx, L[j].gy), -1);
                const Leaf P = L[j];
                for (int c = 0; c < 4; c++) {
                    const int n = (int)L.size();
                    L.push_back({P.level + 1, 2 * P.gx + (c & 1), 2 * P.gy + (c >> 1), P.inst});
                    dead.push_back(0);
                    idx.put(Forest::key(L[n].inst, L[n].level, L[n].gx, L[n].gy), n);
                    check.push_back(n);
                }
            }
        }
        std::vector<Leaf> M;
        M.reserve(L.size());
        for (size_t i = 0; i < L.size(); i++) if (!dead[i]) M.push_back(L[i]);
        L.swap(M);
    }
    if (!changed) {
        bool same = ((int)L.size() == n);
        for (size_t i = 0; same && i < L.size(); i++)
            if (f.lookup(L[i].inst, L[i].level, L[i].gx, L[i].gy) < 0) same = false;
        if (!same) changed = 1;
    }
    return L;
}

std::vector<Leaf> adapt_leaves(const Forest& f, const std::vector<int>& mark, int& changed, std::string& err)
{
    (void)err;
    const int ni = f.ninst(), np = f.np();
    if (ni <= 1) return adapt_patches(f, mark, nullptr, np, changed, true);
    // a batch: the instances on threads, their leaves in instance order
    std::vector<std::vector<int>> list(ni);
    for (int i = 0; i < np; i++) list[f.p[i].inst].push_back(i);
    std::vector<std::vector<Leaf>> out(ni);
    std::vector<int> ch(ni, 0);
    const int nt = std::max(1, std::min((int)std::thread::hardware_concurrency(), 16));
    run_tasks(ni, nt, [&](int k) { out[k] = adapt_patches(f, mark, list[k].data(), (int)list[k].size(), ch[k], false); });
    std::vector<Leaf> L;
    changed = 0;
    for (int k = 0; k < ni; k++) {
        L.insert(L.end(), out[k].begin(), out[k].end());
        changed |= ch[k];
    }
    return L;
}

void smooth_marks(const Forest& f, std::vector<int>& mark, int smooth_level)
{
    const int np = f.np();
    std::vector<int> tl(np);
    for (int i = 0; i < np; i++) tl[i] = f.p[i].level + mark[i];
    for (int i = 0; i < np; i++) {
        const PatchInfo& P = f.p[i];
        const int level = P.level;
        int mt = tl[i];
        // faces first, then corners, each only while no neighbour has raised the target above level
        for (int fc = 0; mt <= level && fc < 4; fc++) {
            const int t = P.face_type[fc];
            if (t == NB_BOUNDARY) continue;
            for (int k = 0; k < (t == NB_HALF ? 2 : 1); k++) {
                const int nb = P.face_nbr[fc][k];
                if (f.p[nb].level + f.gi(f.p[nb].inst).lbase >= smooth_level) mt = std::max(mt, tl[nb]);
            }
        }
        for (int c = 0; mt <= level && c < 4; c++) {
            if (!P.has_corner[c]) continue;
            const int nb = P.corner_nbr[c];
            if (f.p[nb].level + f.gi(f.p[nb].inst).lbase >= smooth_level) mt = std::max(mt, tl[nb]);
        }
        mark[i] = (mt < level) ? -1 : (mt > level) ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// partition along the space-filling curve
// ---------------------------------------------------------------------------
void make_partition(const Forest& f, int rank, int size, PartitionPlan& out)
{
    const int np = f.np();
    out.rank = rank;
    out.size = size;
    out.owner.assign(np, 0);
    // SFC order over all levels: (instance, block, Morton of the lower-left corner at the finest scale)
    std::vector<int> sfc(np);
    for (int i = 0; i < np; i++) sfc[i] = i;
    std::sort(sfc.begin(), sfc.end(), [&](int a, int b) {
        const PatchInfo &A = f.p[a], &B = f.p[b];
        if (A.inst != B.inst) return A.inst < B.inst;
        if (A.block != B.block) return A.block < B.block;
        return A.morton < B.morton;
    });
    // weight: substeps per coarse step; a leaf goes to the rank whose share of the
    // total weight holds the middle of the leaf's weight interval
    const int lmin = f.minlevel_present;
    double W = 0.0;
    for (int i = 0; i < np; i++) W += std::ldexp(1.0, f.p[i].level - lmin);
    double cw = 0.0;
    for (int k = 0; k < np; k++) {
        const int i = sfc[k];
        const double w = std::ldexp(1.0, f.p[i].level - lmin);
        const int r = (int)std::floor((cw + 0.5 * w) * size / W);
        out.owner[i] = std::min(std::max(r, 0), size - 1);
        cw += w;
    }
    // neighbours across faces and corners
    auto nbrs = [&](int i, std::vector<int>& v) {
        v.clear();
        const PatchInfo& P = f.p[i];
        for (int fc = 0; fc < 4; fc++) {
            if (P.face_type[fc] == NB_BOUNDARY) continue;
            for (int k = 0; k < (P.face_type[fc] == NB_HALF ? 2 : 1); k++) v.push_back(P.face_nbr[fc][k]);
        }
        for (int c = 0; c < 4; c++)
            if (P.has_corner[c]) v.push_back(P.corner_nbr[c]);
    };
    // ring[r][i]: 1 (ring 1) or 2 (ring 2) of rank r, for patches r does not own
    std::vector<std::vector<char>> ring(size, std::vector<char>(np, 0));
    std::vector<int> nb;
    for (int i = 0; i < np; i++) {
        nbrs(i, nb);
        for (int j : nb)
            if (out.owner[j] != out.owner[i]) ring[out.owner[i]][j] = 1;
    }
    for (int r = 0; r < size; r++)
        for (int i = 0; i < np; i++) {
            if (ring[r][i] != 1) continue;
            nbrs(i, nb);
            for (int j : nb)
                if (out.owner[j] != r && ring[r][j] == 0) ring[r][j] = 2;
        }
    out.fill.assign(np, 0);
    for (int i = 0; i < np; i++) out.fill[i] = (out.owner[i] == rank || ring[rank][i] == 1) ? 1 : 0;
    out.peers.clear(); out.send.clear(); out.recv.clear();
    for (int r = 0; r < size; r++) {
        if (r == rank) continue;
        std::vector<int> snd, rcv;
        for (int i = 0; i < np; i++) {
            if (out.owner[i] == rank && ring[r][i]) snd.push_back(i);
            if (out.owner[i] == r && ring[rank][i]) rcv.push_back(i);
        }
        if (snd.empty() && rcv.empty()) continue;
        out.peers.push_back(r);
        out.send.push_back(snd);
        out.recv.push_back(rcv);
    }
    // owned slots of each level: one range, since a level's slots follow the SFC order
    for (int l = 0; l < 34; l++) { out.own_lo[l] = 0; out.own_hi[l] = 0; }
    for (int l = 0; l < 33; l++) {
        int lo = -1, hi = -1;
        for (int i = f.lev_off[l]; i < f.lev_off[l + 1]; i++)
            if (out.owner[i] == rank) { if (lo < 0) lo = i; hi = i + 1; }
        if (lo >= 0) { out.own_lo[l] = lo; out.own_hi[l] = hi; }
        else { out.own_lo[l] = out.own_hi[l] = f.lev_off[l]; }
    }
}

// ---------------------------------------------------------------------------
// gather tables
// ---------------------------------------------------------------------------
namespace {

struct TableCtx {
    const Forest& f;
    int mx, my, mbc, nx, nq;
    bool sph;
    TableCtx(const Forest& ff) : f(ff)
    {
        mx = ff.g.d.mx; my = ff.g.d.my; mbc = ff.g.d.mbc; nx = mx + 2 * mbc; nq = ff.g.d.nq();
        sph = ff.sphere();
    }
    // absolute offset of Fortran cell (i,j), field 0, of slot p
    int cell(int p, int i, int j) const { return p * nq + (j + mbc - 1) * nx + (i + mbc - 1); }
    // block and cell origin of a patch at its level: brick-global for bricks (one
    // coordinate system), block-local for the cubed sphere
    void org(const PatchInfo& P, int& b, long& X0, long& Y0) const
    {
        if (!sph) { b = 0; X0 = (long)P.gx * mx; Y0 = (long)P.gy * my; return; }
        const long n = 1L << P.level;
        b = (int)(P.gx / n);
        X0 = (P.gx - b * n) * mx;
        Y0 = (long)P.gy * my;
    }
    // cell (X, Y) of block b at level L in the coordinates of block b2 (adjacent or equal)
    void to_block(int b, int b2, int L, long X, long Y, long& X2, long& Y2) const
    {
        if (b == b2) { X2 = X; Y2 = Y; return; }
        const int fc = cs_face_to(b, b2);
        if (fc < 0) { X2 = Y2 = -(1L << 20); return; }   // not adjacent: outside every patch (tables check)
        cs_xform(b, fc, (long)mx << L, X, Y, X2, Y2);
    }
    // An index map (x, y) -> (c + M (x, y)) with integer M.  to_block is the identity
    // or an isometry of the plane between adjacent blocks (a constant outside point
    // otherwise), so the transforms below are affine and three evaluations give them.
    struct Aff {
        long ci, cj, ii, ij, ji, jj;
        void map(long x, long y, int& i2, int& j2) const
        {
            i2 = (int)(ci + ii * x + ij * y);
            j2 = (int)(cj + ji * x + jj * y);
        }
    };
    // transform_face / transform_corner: cell (i, j) of P as a Fortran index of N, same level
    void same(const PatchInfo& P, long i, long j, const PatchInfo& N, long& i2, long& j2) const
    {
        int b, bn; long X0, Y0, XN, YN, X2, Y2;
        org(P, b, X0, Y0); org(N, bn, XN, YN);
        to_block(b, bn, P.level, X0 + i - 1, Y0 + j - 1, X2, Y2);
        i2 = X2 - XN + 1; j2 = Y2 - YN + 1;
    }
    Aff same_map(const PatchInfo& P, const PatchInfo& N) const
    {
        long a0, b0, a1, b1, a2, b2;
        same(P, 0, 0, N, a0, b0); same(P, 1, 0, N, a1, b1); same(P, 0, 1, N, a2, b2);
        return {a0, b0, a1 - a0, a2 - a0, b1 - b0, b2 - b0};
    }
    // transform_face2 / transform_corner2: child (a, c) -- in the coarse patch's axes -- of
    // coarse cell (i, j) of C, as a Fortran index of the fine patch F; affine in
    // (x, y) = (2 i + a, 2 j + c)
    void child(const PatchInfo& C, long x, long y, const PatchInfo& F, long& i2, long& j2) const
    {
        int b, bf; long X0, Y0, XF, YF, X2, Y2;
        org(C, b, X0, Y0); org(F, bf, XF, YF);
        to_block(b, bf, C.level + 1, 2 * (X0 - 1) + x, 2 * (Y0 - 1) + y, X2, Y2);
        i2 = X2 - XF + 1; j2 = Y2 - YF + 1;
    }
    Aff child_map(const PatchInfo& C, const PatchInfo& F) const
    {
        long a0, b0, a1, b1, a2, b2;
        child(C, 0, 0, F, a0, b0); child(C, 1, 0, F, a1, b1); child(C, 0, 1, F, a2, b2);
        return {a0, b0, a1 - a0, a2 - a0, b1 - b0, b2 - b0};
    }
};

}  // namespace

// Every gather index must lie in the q slab, or a wrong transform would send the ghost-fill
// kernels outside it: copy and average ops are checked as they are made, interpolation and
// physical-BC entries as they are concatenated.
bool build_tables(const Forest& f, const int mthbc[4], bool inflow, Tables& out, TableWork& w, std::string& err)
{
    TableCtx T(f);
    const int mx = T.mx, my = T.my, mbc = T.mbc, nq = T.nq, np = f.np();
    const int nxy = T.nx * (my + 2 * mbc);
    int nt = (int)std::thread::hardware_concurrency();
    nt = std::max(1, std::min(nt, std::min(16, np / 64)));
    int nlev = 0;
    for (int l = 0; l < 33; l++) if (f.lev_off[l + 1] > f.lev_off[l]) nlev = l + 1;
    std::atomic<int> bad{0};

    // ---- copy2ghost (faces, then corners, of each patch: fclaw2d_clawpatch46_copy.f) and
    // ---- average2ghost (coarse = this patch: faces, then corners) as region ops ----
    // The ghost-fill kernel enumerates each op's cells and applies its map.  Copy
    // destinations (the four face strips along 1..mx or 1..my and the four corner
    // blocks) are disjoint, each face or corner has one same-size neighbour, and the
    // children of one coarse ghost cell lie in one of the two half-size neighbours of
    // its face, so no cell is written twice and the ops' order does not matter.
    auto in_box = [&](int i, int j) { return 1 - mbc <= i && i <= mx + mbc && 1 - mbc <= j && j <= my + mbc; };
    auto region_box = [&](int region, int& ilo, int& ihi, int& jlo, int& jhi) {
        if (region == 0) { ilo = 1 - mbc; ihi = 0; jlo = 1; jhi = my; }
        else if (region == 1) { ilo = mx + 1; ihi = mx + mbc; jlo = 1; jhi = my; }
        else if (region == 2) { ilo = 1; ihi = mx; jlo = 1 - mbc; jhi = 0; }
        else if (region == 3) { ilo = 1; ihi = mx; jlo = my + 1; jhi = my + mbc; }
        else {
            const int cr = region - 4;
            ilo = (cr & 1) ? mx + 1 : 1 - mbc; ihi = ilo + mbc - 1;
            jlo = (cr & 2) ? my + 1 : 1 - mbc; jhi = jlo + mbc - 1;
        }
    };
    auto op = [](int dst, int src, int region, const TableCtx::Aff& A) {
        return FillOp{dst, src, region, 0, (int)A.ci, (int)A.cj, (int)A.ii, (int)A.ij, (int)A.ji, (int)A.jj};
    };
    // a copy region's sources: the map is affine, so the region's four corner cells
    // bound them; all must lie in the source patch (with its ghost cells)
    auto copy_ok = [&](int region, const TableCtx::Aff& A) {
        int ilo, ihi, jlo, jhi, i2, j2;
        region_box(region, ilo, ihi, jlo, jhi);
        for (int c = 0; c < 4; c++) {
            A.map((c & 1) ? ihi : ilo, (c & 2) ? jhi : jlo, i2, j2);
            if (!in_box(i2, j2)) return false;
        }
        return true;
    };
    // an average corner's children (its face ops keep only cells whose children are
    // interior cells of the fine patch, in the kernel)
    auto avg_corner_ok = [&](int region, const TableCtx::Aff& F) {
        int ilo, ihi, jlo, jhi, i2, j2;
        region_box(region, ilo, ihi, jlo, jhi);
        for (int jc = jlo; jc <= jhi; jc++)
            for (int ic = ilo; ic <= ihi; ic++)
                for (int m = 0; m < 4; m++) {
                    F.map(2 * ic + (m & 1), 2 * jc + (m >> 1), i2, j2);
                    if (!in_box(i2, j2)) return false;
                }
        return true;
    };
    // ---- the tables of each patch: region ops, physical BCs, time-interpolation list and
    // time-sync ops, in chunks of up to 64 patches of one level (one task each) ----
    struct PChunk { int l, a, b; };
    std::vector<PChunk> pch;
    for (int l = 0; l < nlev; l++)
        for (int a = f.lev_off[l]; a < f.lev_off[l + 1]; a += 64) pch.push_back({l, a, std::min(f.lev_off[l + 1], a + 64)});
    w.copy.resize(pch.size()); w.avg.resize(pch.size()); w.phys.resize(pch.size()); w.ti.resize(pch.size());
    out.sync.resize((size_t)np * SYNC_SLOTS);           // every slot is written by its patch's task
    auto phys_sync = [&](int c) {
        const int a0 = pch[c].a, a1 = pch[c].b;
        // ---- setphysical: clawpack46_bc2_default with chains resolved per patch ----
        {
            std::vector<int> wsrc(nxy, -1), wneg(nxy, 0), wconst(nxy, 0);
            for (int ip = a0; ip < a1; ip++) {
                const PatchInfo& P = f.p[ip];
                if (!(P.phys[0] || P.phys[1] || P.phys[2] || P.phys[3])) continue;
                // written cell -> (source cell, negate mask), within this bc2 call;
                // indexed by the plane-0 offset of the cell inside the patch
                const int base = T.cell(ip, 1 - mbc, 1 - mbc);
                std::fill(wsrc.begin(), wsrc.end(), -1);
                std::vector<int> order;
                auto put = [&](int di, int dj, int si, int sj, int neg) {
                    const int dst = T.cell(ip, di, dj);
                    int src = T.cell(ip, si, sj), cst = 0;
                    if (wsrc[src - base] >= 0) { neg ^= wneg[src - base]; cst = wconst[src - base]; src = wsrc[src - base]; }
                    if (wsrc[dst - base] < 0) order.push_back(dst);
                    wsrc[dst - base] = src;
                    wneg[dst - base] = neg;
                    wconst[dst - base] = cst;
                };
                auto put_const = [&](int di, int dj) {
                    const int dst = T.cell(ip, di, dj);
                    if (wsrc[dst - base] < 0) order.push_back(dst);
                    wsrc[dst - base] = dst;
                    wneg[dst - base] = 0;
                    wconst[dst - base] = 1;
                };
                const int NEG2 = 1 << 1, NEG3 = 1 << 2;   // field 2 (x momentum) / field 3 (y momentum)
                int bc[4];
                for (int k = 0; k < 4; k++) bc[k] = P.phys[k] ? mthbc[k] : -1;
                if (bc[0] == 0 && inflow) for (int ibc = 1; ibc <= mbc; ibc++) for (int j = 1 - mbc; j <= my + mbc; j++) put_const(1 - ibc, j);
                if (bc[0] == 1) for (int ibc = 1; ibc <= mbc; ibc++) for (int j = 1 - mbc; j <= my + mbc; j++) put(1 - ibc, j, 1, j, 0);
                if (bc[0] == 3) for (int ibc = 1; ibc <= mbc; ibc++) for (int j = 1 - mbc; j <= my + mbc; j++) put(1 - ibc, j, ibc, j, NEG2);
                if (bc[1] == 1) for (int ibc = 1; ibc <= mbc; ibc++) for (int j = 1 - mbc; j <= my + mbc; j++) put(mx + ibc, j, mx, j, 0);
                if (bc[1] == 3) for (int ibc = 1; ibc <= mbc; ibc++) for (int j = 1 - mbc; j <= my + mbc; j++) put(mx + ibc, j, mx + 1 - ibc, j, NEG2);
                if (bc[2] == 1) for (int jbc = 1; jbc <= mbc; jbc++) for (int i = 1 - mbc; i <= mx + mbc; i++) put(i, 1 - jbc, i, 1, 0);
                if (bc[2] == 3) for (int jbc = 1; jbc <= mbc; jbc++) for (int i = 1 - mbc; i <= mx + mbc; i++) put(i, 1 - jbc, i, jbc, NEG3);
                if (bc[3] == 1) for (int jbc = 1; jbc <= mbc; jbc++) for (int i = 1 - mbc; i <= mx + mbc; i++) put(i, my + jbc, i, my, 0);
                if (bc[3] == 3) for (int jbc = 1; jbc <= mbc; jbc++) for (int i = 1 - mbc; i <= mx + mbc; i++) put(i, my + jbc, i, my + 1 - jbc, NEG3);
                for (int dst : order) w.phys[c].push_back({dst, wsrc[dst - base], wneg[dst - base], wconst[dst - base]});
            }
        }
        // ---- time interpolation patches ----
        for (int ip = a0; ip < a1; ip++) if (f.p[ip].has_fine_nbr) w.ti[c].push_back(ip);
        // ---- time sync ops ----
        // fclaw2d_time_sync applies the same-size corrections of every synced level,
        // then the fine-to-coarse ones (src/fclaw2d_time_sync.c:118-202); each
        // correction adds to cells of its own patch p only and reads registers no
        // correction writes, so per patch the samesize ops (faces 0..3) followed by
        // the f2c ops ((face, igrid) order) give every cell its additions in the
        // reference's order.  Levels without finer neighbours have no f2c ops, so
        // one range of levels [a, maxlevel] covers both kinds.  A patch has at most
        // eight ops (one samesize or two f2c per face): slots 8 p .. 8 p + 7.
        for (int ip = a0; ip < a1; ip++) {
            const PatchInfo& P = f.p[ip];
            SyncOp* slot = &out.sync[(size_t)ip * SYNC_SLOTS];
            int nops = 0;
            for (int fc = 0; fc < 4; fc++)
                if (P.face_type[fc] == NB_SAME && (!f.sphere() || f.p[P.face_nbr[fc][0]].block == P.block))
                    slot[nops++] = {ip, P.face_nbr[fc][0], fc, 0, 0, SYNC_SAMESIZE, {0, 0}};
            for (int fc = 0; fc < 4; fc++) {
                if (P.face_type[fc] != NB_HALF) continue;
                if (f.sphere() && f.p[P.face_nbr[fc][0]].block != P.block) continue;
                for (int ig = 0; ig < 2; ig++) {
                    const int fi = P.face_nbr[fc][ig];
                    const PatchInfo& F = f.p[fi];
                    const int noff = (fc < 2) ? (2 * P.gy - F.gy) * my : (2 * P.gx - F.gx) * mx;
                    slot[nops++] = {ip, fi, fc, ig, noff, SYNC_F2C, {0, 0}};
                }
            }
            for (; nops < SYNC_SLOTS; nops++) slot[nops] = SyncOp{0, 0, 0, 0, 0, SYNC_NONE, {0, 0}};
        }
    };
    auto patches = [&](int c) {
        std::vector<FillOp>& vc = w.copy[c];
        std::vector<FillOp>& va = w.avg[c];
        vc.clear(); va.clear(); w.phys[c].clear(); w.ti[c].clear();
        bool good = true;
        for (int ip = pch[c].a; ip < pch[c].b; ip++) {
            const PatchInfo& P = f.p[ip];
            for (int fc = 0; fc < 4; fc++) {
                if (P.face_type[fc] != NB_SAME) continue;
                const int n = P.face_nbr[fc][0];
                const TableCtx::Aff A = T.same_map(P, f.p[n]);
                good = good && copy_ok(fc, A);
                vc.push_back(op(ip, n, fc, A));
            }
            for (int cr = 0; cr < 4; cr++) {
                if (!P.has_corner[cr] || P.corner_type[cr] != NB_SAME) continue;
                const int n = P.corner_nbr[cr];
                const TableCtx::Aff A = T.same_map(P, f.p[n]);
                good = good && copy_ok(4 + cr, A);
                vc.push_back(op(ip, n, 4 + cr, A));
            }
            if (!P.on_cf) continue;
            for (int fc = 0; fc < 4; fc++) {
                if (P.face_type[fc] != NB_HALF) continue;
                for (int ig = 0; ig < 2; ig++) {
                    const int fi = P.face_nbr[fc][ig];
                    va.push_back(op(ip, fi, fc, T.child_map(P, f.p[fi])));
                }
            }
            for (int cr = 0; cr < 4; cr++) {
                if (!P.has_corner[cr] || P.corner_type[cr] != NB_HALF) continue;
                const int fi = P.corner_nbr[cr];
                const TableCtx::Aff F = T.child_map(P, f.p[fi]);
                good = good && avg_corner_ok(4 + cr, F);
                va.push_back(op(ip, fi, 4 + cr, F));
            }
        }
        phys_sync(c);
        if (!good) bad = 1;
    };

    // ---- interpolate2ghost (coarse = level l): faces of all coarse patches, then corners ----
    // Two writes to one fine ghost cell come from ops into the same fine patch, so the
    // last-writer rule of the reference's order (faces of every coarse patch in patch
    // order, then corners) is kept per fine patch: the ops are listed per fine patch in
    // that order (one pass here), then the fine patches are expanded in parallel chunks,
    // each with a map of one patch's cells.
    w.iops.resize(33); w.iop_first.resize(33);
    struct Chunk { int l, a, b; };                       // fine patches [a, b) of coarse level l
    std::vector<Chunk> chunks;
    for (int l = 0; l < 32; l++) {
        std::vector<InterpOp>& ops = w.iops[l];
        std::vector<int>& first = w.iop_first[l];
        ops.clear();
        const int p0 = f.lev_off[l], p1 = f.lev_off[l + 1], nf = f.lev_off[l + 2] - p1;
        first.assign(nf + 1, 0);
        if (p0 == p1 || nf == 0) continue;
        auto iop = [&](int cp, int fp, int region) {
            const TableCtx::Aff F = T.child_map(f.p[cp], f.p[fp]);
            return InterpOp{cp, fp, region, 0, F.ci, F.cj, F.ii, F.ij, F.ji, F.jj};
        };
        for (int pass = 0; pass < 2; pass++) {           // count, then fill, in the reference's order
            std::vector<int> at(first.begin(), first.end() - 1);
            auto add = [&](int cp, int fp, int region) {
                if (fp < p1 || fp >= p1 + nf) { bad = 1; return; }
                if (pass == 0) first[fp - p1 + 1]++;
                else ops[at[fp - p1]++] = iop(cp, fp, region);
            };
            for (int ip = p0; ip < p1; ip++) {
                const PatchInfo& C = f.p[ip];
                if (!C.on_cf) continue;
                for (int fc = 0; fc < 4; fc++)
                    if (C.face_type[fc] == NB_HALF)
                        for (int ig = 0; ig < 2; ig++) add(ip, C.face_nbr[fc][ig], fc);
            }
            for (int ip = p0; ip < p1; ip++) {
                const PatchInfo& C = f.p[ip];
                if (!C.on_cf) continue;
                for (int cr = 0; cr < 4; cr++)
                    if (C.has_corner[cr] && C.corner_type[cr] == NB_HALF) add(ip, C.corner_nbr[cr], 4 + cr);
            }
            if (pass == 0) {
                for (int k = 0; k < nf; k++) first[k + 1] += first[k];
                ops.resize(first[nf]);
            }
        }
        for (int a = 0; a < nf; a += 64) chunks.push_back({l, a, std::min(nf, a + 64)});
    }
    w.interp.resize(chunks.size());
    auto interp = [&](int c) {
        const Chunk& ch = chunks[c];
        const int l = ch.l, p1 = f.lev_off[l + 1];
        std::vector<InterpEnt>& v = w.interp[c];
        v.clear();
        std::vector<int> at(nxy, -1);                    // cell of the current fine patch -> entry
        auto validi = [&](long i, long j) { return 1 - mbc <= i && i <= mx + mbc && 1 - mbc <= j && j <= my + mbc; };
        bool outside = false;
        for (int k = ch.a; k < ch.b; k++) {
            const int fp = p1 + k;
            const size_t v0 = v.size();
            // the fine cells of the four children (coarse axes, sub = ii + 2 jj) of coarse
            // cell (ic, jc), skipped unless all lie in the fine patch's padded patch
            // (is_valid_interp)
            auto emit = [&](const InterpOp& o, int ic, int jc, bool check) {
                long ci[4], cj[4];
                for (int m = 0; m < 4; m++) {
                    const long x = 2 * ic + (m & 1), y = 2 * jc + (m >> 1);
                    ci[m] = o.ci + o.ii * x + o.ij * y;
                    cj[m] = o.cj + o.ji * x + o.jj * y;
                    if (check && !validi(ci[m], cj[m])) return;
                }
                for (int m = 0; m < 4; m++) {
                    if (!validi(ci[m], cj[m])) { outside = true; return; }
                    const InterpEnt e{T.cell(fp, (int)ci[m], (int)cj[m]), T.cell(o.cp, ic, jc), m, 0};
                    int& a = at[e.dst - fp * nq];
                    if (a < 0) { a = (int)v.size(); v.push_back(e); }
                    else v[a] = e;
                }
            };
            for (int q = w.iop_first[l][k]; q < w.iop_first[l][k + 1]; q++) {
                const InterpOp& o = w.iops[l][q];
                if (o.region < 2) {
                    for (int ibc = 1; ibc <= mbc / 2; ibc++) {
                        const int ic = (o.region == 0) ? ibc : mx - ibc + 1;
                        for (int jc = 1; jc <= mx; jc++) emit(o, ic, jc, true);
                    }
                } else if (o.region < 4) {
                    for (int jbc = 1; jbc <= mbc / 2; jbc++) {
                        const int jc = (o.region == 2) ? jbc : my - jbc + 1;
                        for (int ic = 1; ic <= mx; ic++) emit(o, ic, jc, true);
                    }
                } else {
                    const int cr = o.region - 4;
                    for (int ibc = 1; ibc <= mbc / 2; ibc++)
                        for (int jbc = 1; jbc <= mbc / 2; jbc++)
                            emit(o, (cr & 1) ? mx - ibc + 1 : ibc, (cr & 2) ? my - jbc + 1 : jbc, false);
                }
            }
            for (size_t i = v0; i < v.size(); i++) at[v[i].dst - fp * nq] = -1;
        }
        if (outside) bad = 1;
    };
    // the interpolation chunks first, then the per-patch chunks
    const int nchunk = (int)chunks.size(), npch = (int)pch.size();
    run_tasks(nchunk + npch, nt, [&](int k) {
        if (k < nchunk) interp(k);
        else patches(k - nchunk);
    });
    if (bad) { err = "a ghost-fill table writes outside its destination patches"; return false; }

    // flat tables in level order (the chunks of a level are consecutive): each chunk's
    // place from prefix sums, then the chunks copied there, and their entries checked
    // against the patches, on the worker threads
    std::vector<size_t> oc(npch + 1, 0), oa(npch + 1, 0), oph(npch + 1, 0), oti(npch + 1, 0), oi(nchunk + 1, 0);
    for (int c = 0; c < npch; c++) {
        oc[c + 1] = oc[c] + w.copy[c].size();
        oa[c + 1] = oa[c] + w.avg[c].size();
        oph[c + 1] = oph[c] + w.phys[c].size();
        oti[c + 1] = oti[c] + w.ti[c].size();
    }
    for (int c = 0; c < nchunk; c++) oi[c + 1] = oi[c] + w.interp[c].size();
    for (int l = 0, c = 0, ci = 0; l < 34; l++) {
        out.copy_off[l] = (int)oc[c];
        out.avg_off[l] = (int)oa[c];
        out.phys_off[l] = (int)oph[c];
        out.ti_off[l] = (int)oti[c];
        out.interp_off[l] = (int)oi[ci];
        while (c < npch && pch[c].l == l) c++;
        while (ci < nchunk && chunks[ci].l == l) ci++;
    }
    // (no clear first: a vector that shrinks or keeps its size is not refilled with zeros)
    out.copy.resize(oc[npch]); out.avg.resize(oa[npch]); out.phys.resize(oph[npch]); out.ti.resize(oti[npch]);
    out.interp.resize(oi[nchunk]);
    const long nall = (long)np * nq;
    auto in_all = [&](long k) { return k >= 0 && k < nall; };
    run_tasks(nchunk + npch, nt, [&](int k) {
        bool good = true;
        if (k < nchunk) {
            std::copy(w.interp[k].begin(), w.interp[k].end(), out.interp.begin() + oi[k]);
            for (const InterpEnt& e : w.interp[k]) good = good && in_all(e.dst) && in_all(e.src) && e.sub >= 0 && e.sub < 4;
        } else {
            const int c = k - nchunk;
            std::copy(w.copy[c].begin(), w.copy[c].end(), out.copy.begin() + oc[c]);
            std::copy(w.avg[c].begin(), w.avg[c].end(), out.avg.begin() + oa[c]);
            std::copy(w.phys[c].begin(), w.phys[c].end(), out.phys.begin() + oph[c]);
            std::copy(w.ti[c].begin(), w.ti[c].end(), out.ti.begin() + oti[c]);
            for (const PhysEnt& e : w.phys[c]) good = good && in_all(e.dst) && in_all(e.src);
        }
        if (!good) bad = 1;
    });
    if (bad) {
        err = "a ghost-fill table indexes outside the patches (bad transform)";
        return false;
    }
    return true;
}

}  // namespace fcb
