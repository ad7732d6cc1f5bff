// host_forest.hpp -- host-side forest of patches and the device gather tables.
//
// The forest plays p4est's role for the B200 package: leaves of a quadtree over
// a brick of equally oriented blocks or over the six blocks of the cubed sphere
// (faces joined with rotations), face/corner neighbour relations, 2:1
// face+corner balance and adaptation.  From it the host builds, once per
// regrid, the per-level gather tables that turn the reference's per-patch
// ghost-fill and time-sync callbacks into single device launches.
#pragma once
#include <stdint.h>
#include <string>
#include <unordered_map>
#include <functional>
#include <vector>
#include "kernels.h"

namespace fcb {

enum { NB_BOUNDARY = 0, NB_HALF = 1, NB_SAME = 2, NB_DOUBLE = 3 };

// level: forest level (the instance's refinement level minus its lbase); gx, gy:
// integer patch coordinates over the instance's brick at its refinement level.
struct Leaf { int level, gx, gy; int inst = 0; };

// Cubed-sphere connectivity, derived from the mapping (fcb_sphere.h): face f of
// block b touches face nf of block nb; a point (x, y) of block b's coordinates
// (inside or beyond face f) is (x', y') = M (x, y) + c in block nb's coordinates.
struct CSFace { int nb, nf, flip; int M[2][2]; int c[2]; };
const CSFace& cs_face(int b, int f);
// Cell (or patch) (X, Y) of block b at N cells per block side, in block nb = cs_face(b, f).nb.
void cs_xform(int b, int f, long N, long X, long Y, long& X2, long& Y2);
// The face of block a whose neighbour is block b (-1: not adjacent, or a == b).
int cs_face_to(int a, int b);

// Open-addressing map from 64-bit keys (Forest::key) to slots, for the lookups of
// neighbour searches and balance: linear probing over a power-of-two table.
class KeyIndex {
public:
    void reset(size_t n)
    {
        size_t cap = 16;
        while (cap < 2 * n + 16) cap <<= 1;
        keys_.assign(cap, EMPTY);
        vals_.assign(cap, -1);
        mask_ = cap - 1;
    }
    void put(uint64_t k, int v)
    {
        size_t h = hash(k);
        while (keys_[h] != EMPTY && keys_[h] != k) h = (h + 1) & mask_;
        keys_[h] = k;
        vals_[h] = v;
    }
    int get(uint64_t k) const
    {
        if (keys_.empty()) return -1;
        size_t h = hash(k);
        while (keys_[h] != EMPTY) {
            if (keys_[h] == k) return vals_[h];
            h = (h + 1) & mask_;
        }
        return -1;
    }
private:
    static constexpr uint64_t EMPTY = ~0ull;
    size_t hash(uint64_t k) const { return (size_t)((k * 0x9E3779B97F4A7C15ull) >> 17) & mask_; }
    std::vector<uint64_t> keys_;
    std::vector<int> vals_;
    size_t mask_ = 0;
};

struct PatchInfo {
    int level, gx, gy, block;
    int inst;
    uint64_t morton;
    double xlower, ylower, dx, dy;
    int face_type[4];
    int face_nbr[4][2];
    int phys[4];
    int has_corner[4], corner_type[4], corner_nbr[4];
    int bcc3[4];      // corner c is a corner of the cubed sphere (three blocks meet, no corner neighbour)
    int has_fine_nbr, on_cf;
};

struct Geometry {
    Dims d;
    int mi, mj;
    double ax, bx, ay, by;
    int lbase = 0;    // refinement level of forest level 0 (an instance's minlevel in a batch)
    int kind = 0;     // 0: brick of mi x mj equally oriented blocks; 1: cubed sphere (6 blocks, gx = block 2^l + ix)
};

class Forest {
public:
    Geometry g;                      // the single domain, or instance 0
    std::vector<Geometry> inst;      // per-instance domains of a batch (empty: one domain, g)
    std::vector<PatchInfo> p;        // slot order: level-major, then instance, block, Morton
    int lev_off[34];                 // patches of level l: [lev_off[l], lev_off[l+1])
    int minlevel_present = 0, maxlevel_present = -1;

    // Install leaves (any order).  Returns false (and sets err) if not 2:1 balanced.
    bool build(const std::vector<Leaf>& leaves, std::string& err);
    int lookup(int l, int x, int y) const { return lookup(0, l, x, y); }
    int lookup(int i, int l, int x, int y) const;
    int np() const { return (int)p.size(); }
    int ninst() const { return inst.empty() ? 1 : (int)inst.size(); }
    const Geometry& gi(int i) const { return inst.empty() ? g : inst[i]; }
    bool in_domain(int l, int x, int y) const { return in_domain(0, l, x, y); }
    bool in_domain(int i, int l, int x, int y) const
    {
        const Geometry& G = gi(i);
        const int la = l + G.lbase;
        return l >= 0 && x >= 0 && y >= 0 && x < (G.mi << la) && y < (G.mj << la);
    }
    void geometry(PatchInfo& q) const;
    bool sphere(int i = 0) const { return gi(i).kind == 1; }
    // Patch (x, y) of level l stepped by (dx, dy), |dx|, |dy| <= 1, across block faces:
    // 1 with the neighbour position in (ox, oy); 0 outside the domain (physical boundary);
    // -1 across a cubed-sphere corner (no diagonal neighbour there).
    int step(int i, int l, int x, int y, int dx, int dy, int& ox, int& oy) const;
    static uint64_t key(int i, int l, int x, int y)
    {
        return ((uint64_t)i << 56) | ((uint64_t)l << 50) | ((uint64_t)x << 25) | (uint64_t)y;
    }

private:
    KeyIndex index_;
    std::vector<PatchInfo> scratch_;   // leaves with their geometry, before the slot order
};

// Refine marked leaves, coarsen fully marked families, then 2:1 balance
// (p4est_wrap adapt semantics).  mark: +1 refine, -1 coarsen, 0 keep.
// Returns the new leaf list; changed = 0 if identical to the old forest.
std::vector<Leaf> adapt_leaves(const Forest& f, const std::vector<int>& mark, int& changed, std::string& err);

// Refinement smoothing of fclaw2d_domain_adapt (src/fclaw2d_convenience.c:507-645):
// mark (+1 / -1 / 0 from the tags) sets each leaf's target level; every leaf
// then takes the largest target level of itself and its face and corner
// neighbours of level >= smooth_level and is marked by the sign of the
// difference to its own level.
void smooth_marks(const Forest& f, std::vector<int>& mark, int smooth_level);

// Partition of a single forest over ranks along the space-filling curve (p4est's
// leaf order: block, then Morton order) with weight 2^(level - minlevel present) per
// leaf, its number of substeps in a coarse step (src/fclaw2d_partition.c:113 uses
// p4est's weighted partition).  Every rank keeps the whole tree; it owns one SFC
// range, updates its own patches and fills the ghost cells of its own patches and
// of ring 1 (the other ranks' patches touching its own across a face or corner,
// which its interpolations read as coarse sources).  Ring 2 (the patches touching
// ring 1) supplies those fills; rings 1 and 2 make the halo it receives before each
// ghost update.
struct PartitionPlan {
    int rank = 0, size = 1;
    std::vector<int> owner;                  // per slot
    std::vector<char> fill;                  // per slot: owned or ring 1 (ghost cells filled here)
    std::vector<int> peers;                  // ranks this one exchanges with (ascending)
    std::vector<std::vector<int>> send;      // per peer: own slots in the peer's halo (ascending)
    std::vector<std::vector<int>> recv;      // per peer: the peer's slots in this halo (ascending)
    int own_lo[34], own_hi[34];              // owned slots of level l: [own_lo[l], own_hi[l])
};
// The plan of `rank` among `size` ranks for forest f (pure host computation).
void make_partition(const Forest& f, int rank, int size, PartitionPlan& out);

// Ghost-fill tables of a forest, flat in level order: level l's entries of table x are
// x[x_off[l], x_off[l + 1]).
struct Tables {
    std::vector<FillOp> copy;        // copy2ghost(level): region ops of the level's patches
    std::vector<FillOp> avg;         // average2ghost(level): level is the coarse level
    std::vector<InterpEnt> interp;   // interpolate2ghost(level): level is the coarse level
    std::vector<PhysEnt> phys;       // setphysical(level)
    std::vector<int> ti;             // patches with fine-grid neighbours (fclaw2d_timeinterp)
    // time-sync corrections of patch p: sync[SYNC_SLOTS p .. SYNC_SLOTS p + 7], in the
    // reference's order, unused slots SYNC_NONE
    std::vector<SyncOp> sync;
    int copy_off[34], avg_off[34], interp_off[34], phys_off[34], ti_off[34];
};

// Buffers build_tables keeps between calls (their pages stay mapped from one regrid
// to the next).
// One interpolation op of the table build: coarse patch cp fills ghost cells of fine
// patch fp through face (region 0..3) or corner (4..7) of cp; the child map of the pair
// (x, y) -> (ci + ii x + ij y, cj + ji x + jj y).
struct InterpOp { int cp, fp, region, pad; long ci, cj, ii, ij, ji, jj; };
struct TableWork {
    std::vector<std::vector<FillOp>> copy, avg;            // region ops per chunk of patches
    std::vector<std::vector<PhysEnt>> phys;                // physical-BC entries per chunk of patches
    std::vector<std::vector<int>> ti;                      // time-interpolation patches per chunk
    std::vector<std::vector<InterpOp>> iops;               // interpolation ops per coarse level, by fine patch
    std::vector<std::vector<int>> iop_first;               // per coarse level: CSR offsets over its fine patches
    std::vector<std::vector<InterpEnt>> interp;            // interpolation entries per task
};

// fn(0) .. fn(n - 1) on the host worker threads (the caller's among them); returns when all are done.
void parallel_for(int n, const std::function<void(int)>& fn);

// inflow: mthbc = 0 sides are set to a constant state (PhysEnt.cst = 1, src unused).
// False (with err) if a table would index outside the patches.
bool build_tables(const Forest& f, const int mthbc[4], bool inflow, Tables& out, TableWork& w, std::string& err);

}  // namespace fcb
