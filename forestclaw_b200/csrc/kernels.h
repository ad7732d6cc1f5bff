// kernels.h -- host-callable launch wrappers of the device kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "fcb_common.h"
#include "fc2d_b200.h"

namespace fcb {

// Programmatic dependent launch of the advance's kernels (fcb_launch.cuh): set
// for the calling thread while a ProgrammaticScope lives.
void set_programmatic_launch(bool on);
bool programmatic_launch();
struct ProgrammaticScope {
    bool prev;
    explicit ProgrammaticScope(bool on) : prev(programmatic_launch()) { set_programmatic_launch(on); }
    ~ProgrammaticScope() { set_programmatic_launch(prev); }
};

struct Dims {
    int mx, my, mbc, meqn, maux;
    int nx() const { return mx + 2 * mbc; }
    int ny() const { return my + 2 * mbc; }
    int nxy() const { return nx() * ny(); }
    int nq() const { return nxy() * meqn; }
    int naux() const { return nxy() * maux; }
    // conservation registers per patch (fclaw2d_clawpatch_conservation.h:56-77)
    int nreg() const { return 4 * my * meqn + 4 * mx * meqn + 4 * my * meqn + 4 * mx * meqn; }
    // cell areas of a manifold patch cover -mbc..mx+mbc+1 (one ring more than q)
    int narea() const { return (mx + 2 * mbc + 2) * (my + 2 * mbc + 2); }
};

// ---- fused update (k_step2_<precision>_<family>.cu) ---------------------------
// Each unit holds a table of launchers, one per (solver, patch size, patch-to-CTA
// mapping); the first entry of a shape is its default.  A launcher called with
// npatch = 0 only sets the kernel's shared-memory attribute.  A launch covers
// lg.nlev consecutive levels; the patches of its k-th level (ascending, from
// relative patch lg.start[k]) take sp[lg.nlev - 1 - k] (the parameter blocks are
// in issue order, finest level first).  The split is a kernel argument, so no
// patch reads memory to find its parameters.
typedef cudaError_t (*Step2Fn)(double* q, double* qlast, const double* aux, double* regs, const PatchDesc* desc,
                               int p0, int npatch, const StepParams* sp, const LevelGroup& lg,
                               unsigned long long* cfl_bits,
                               cudaStream_t st);
struct Step2Variant {
    int precision, rp, mx, my, mbc;
    int threads, min_blocks;   // CTA size and __launch_bounds__ occupancy target
    int reg;                   // 1: one thread per interface (normal solve kept in registers)
    int smem;                  // dynamic shared memory per CTA, bytes
    int persistent;            // 1: a grid of resident CTAs loops over the patches
    Step2Fn fn;
    int spec;                  // 0: any method flags; k > 0: a kernel specialised for limiter k (host checks the options)
};
// Layout version of the kernel parameter structs, checked when an application
// registers update kernels compiled in its own module (include/fc2d_b200_user.cuh).
constexpr int device_abi()
{
    return 1000000 + 1000 * (int)sizeof(StepParams) + 10 * (int)sizeof(PatchDesc) + (int)(sizeof(LevelGroup) % 10);
}
const Step2Variant* step2_table_f64_adv(int* n);
const Step2Variant* step2_table_f64_sw(int* n);
const Step2Variant* step2_table_f64_euler(int* n);
const Step2Variant* step2_table_f32w_adv(int* n);
const Step2Variant* step2_table_f32w_sw(int* n);
const Step2Variant* step2_table_f32w_euler(int* n);

// ---- ghost fill (k_amr.cu) ----------------------------------------------------
// Gather tables: offsets are absolute indices of field 0 in the q slab; fields
// follow at +m*nxy.
// Copy and average run from region ops instead: one op fills the ghost cells of patch
// `dst` on one face (region 0..3: x-low, x-high, y-low, y-high) or corner (4..7: 4 + cr,
// cr = 1 * (x-high) + 2 * (y-high)) from patch `src`, through the integer affine map
// (x, y) -> (ci + ii x + ij y, cj + ji x + jj y) into src's Fortran cell indices:
//   copy     (x, y) = (i, j), a ghost cell of dst; its same-size cell in src
//   average  (x, y) = (2 ic + a, 2 jc + c), child (a, c) -- in dst's axes -- of dst's coarse
//            ghost cell (ic, jc); face ops skip cells whose four children are not all
//            interior cells of src (fclaw2d_clawpatch_is_valid_average)
// A face covers mbc x my (x faces) or mx x mbc (y faces) cells, a corner mbc x mbc.
struct FillOp { int dst, src, region, pad; int ci, cj, ii, ij, ji, jj; };
struct InterpEnt { int dst, src, sub, pad; };      // sub = child position 0..3 (ii + 2 jj)
struct PhysEnt { int dst, src, neg, cst; };        // neg: bit m set => negate field m; cst: constant state

// One table segment of a gather stage: entries e[0..n) from src into dst.
template <class E> struct GatherSeg { double* dst; const double* src; const E* e; int n; };
// average segments and copy segments of one ghost update in one launch (disjoint ghost
// cells); area: per-patch cell areas (one ring more than q per patch) for the
// area-weighted average of a manifold, or null for the plain mean.
void launch_average_copy(const Dims& d, const GatherSeg<FillOp>& a0, const GatherSeg<FillOp>& a1,
                         const GatherSeg<FillOp>& c0, const GatherSeg<FillOp>& c1, const double* area,
                         cudaStream_t st);
void launch_restore_patches(const Dims& d, double* dst, const double* src, const int* slots, int n, cudaStream_t st);
void launch_interp(const Dims& d, const GatherSeg<InterpEnt>& s0, const GatherSeg<InterpEnt>& s1, cudaStream_t st);
void launch_phys(const Dims& d, const GatherSeg<PhysEnt>& s0, const GatherSeg<PhysEnt>& s1, const double* bcstate,
                 cudaStream_t st);
// time interpolation factor of each level (levels 0..31) for a launch over the
// time-interpolation lists of several levels
struct LevelAlpha { double a[32]; };
void launch_timeinterp(const Dims& d, const double* q, const double* qlast, double* qinterp, const int* patches,
                       int npatch, const PatchDesc* desc, const LevelAlpha& alpha, cudaStream_t st);

// ---- time sync (k_amr.cu) -------------------------------------------------------
// One time-sync correction of patch p from neighbour n across face `face`:
// kind SYNC_SAMESIZE (clawpack46_fort_time_sync_samesize) or SYNC_F2C (coarse p,
// fine n = child igrid of the face, n_off = first fine index offset along it).
enum { SYNC_SAMESIZE = 0, SYNC_F2C = 1, SYNC_NONE = -1 };
struct SyncOp { int p, n, face, igrid; int n_off; int kind; int pad[2]; };
constexpr int SYNC_SLOTS = 8;      // ops of a patch: at most one samesize or two f2c per face
// The corrections of a time sync over patches p0 .. p0 + np - 1: the ops of patch p are
// ops[SYNC_SLOTS p ..] (samesize faces 0..3, then f2c ops in (face, igrid) order; the
// rest SYNC_NONE).
void launch_sync(const Dims& d, double* q, const double* regs, const PatchDesc* desc, const SyncOp* ops, int p0,
                 int np, cudaStream_t st);
// All register resets of one fclaw2d_time_sync(minlevel, maxl) call in one launch
// over the patches of levels [minlevel, maxl].
void launch_reset_sync(const Dims& d, double* regs, const PatchDesc* desc, int p0, int np, int minlevel, int maxl,
                       cudaStream_t st);

// ---- diagnostics / regrid (k_amr.cu) -------------------------------------------
// area (manifold, else null): the cell areas weight q instead of dx dy
void launch_patch_mass(const Dims& d, const double* q, const PatchDesc* desc, int np, double* out,
                       cudaStream_t st, const double* area = nullptr);
// Tagging tests of every patch with criterion crit (FC2D_B200_TAG_*, resolved: not TAG_APP) on
// field plane mq: flags[p] bit0 = some cell exceeds refine_thr, bit1 = no cell exceeds coarsen_thr.
// TAG_MINMAX writes the range of the padded patch into minmax (2 doubles per patch), bit0 =
// range > refine_thr, and leaves the family test to the caller.
void launch_tag(const Dims& d, const double* q, const PatchDesc* desc, int np, int crit, int mq, double refine_thr,
                double coarsen_thr, int* flags, cudaStream_t st, double* minmax);
// Halo payload of a partitioned forest: q, qlast and registers of the listed slots,
// nq + nq + nreg doubles per patch, packed into (or unpacked from) one buffer.
void launch_pack_patches(const Dims& d, const int* slots, int n, const double* q, const double* qlast,
                         const double* regs, double* out, cudaStream_t st);
void launch_unpack_patches(const Dims& d, const int* slots, int n, double* q, double* qlast, double* regs,
                           const double* in, cudaStream_t st);
// Repopulation after adapt: op kind 0 copy old slot, 1 interpolate2fine from old parent (igrid),
// 2 average2coarse from 4 old children (src = first child slot; children consecutive by igrid
// via child_slots).
// ---- allocation-free mass (k_mass_noalloc.cu) ------------------------------------
// Capacity of the file-scope device scratch: patch partials (npatches*meqn) plus
// the meqn results must fit.  1 MiB.
enum { MASS_SCRATCH_DOUBLES = 131072 };
// Device address of the scratch on the current device.
cudaError_t mass_scratch_address(double** ptr);
// Partials, then per-field sums at scratch[np*meqn + m]; the stream orders the two launches.
void launch_mass_noalloc(const Dims& d, const double* q, const PatchDesc* desc, int np, double* scratch,
                         cudaStream_t st);

// ---- p*-seed network (k_mlp.cu) ----------------------------------------------------
cudaError_t mlp_setup();
void launch_mlp_blob(const float* prm, void* blob, cudaStream_t st);
void launch_mlp_targets(const double* prim, int n, double gam, double tol, float* X, float* Y, int* iters,
                        cudaStream_t st);
int mlp_fwdbwd_blocks(int nb);
void launch_mlp_step(const float* X, const float* Y, const int* idx, int nb, void* blob, float* prm, float* grad,
                     float* m, float* v, float* partial, float* loss_partial, float* loss, float lr, int step,
                     bool update, unsigned* status, cudaStream_t st);
void launch_mlp_predict(const float* X, int n, const void* blob, float* Y, cudaStream_t st);
// the same evaluation on the tcgen05 tensor cores, 128 states per CTA (k_mlp_tc.cu); a
// tile whose MMAs do not complete sets STATUS_TENSOR in *status and writes nothing
cudaError_t mlp_tc_setup();
void launch_mlp_predict_tc(const float* X, int n, const void* blob, float* Y, unsigned* status, cudaStream_t st);
void launch_mlp_newton_iters(const double* prim, const float* X, const float* Yseed, int n, double gam, double tol,
                             int* iters, cudaStream_t st);
void launch_sample_interfaces(const Dims& d, const double* q, int np, double gam, unsigned long long seed, int n,
                              double* prim, cudaStream_t st);

struct RepopOp { int kind, dst, src, igrid; int child[4]; };
// oarea/narea (cubed sphere, else null): old and new cell areas -- interpolate2fine then
// keeps each coarse cell's mass (fixcapaq2) and average2coarse weights by area.
// aux of the n patches of a new forest from the old slab or staged host values (src codes
// at k_aux_repop)
void launch_aux_repop(const Dims& d, const int* src, int n, const double* oaux, const double* staged, double* aux,
                      cudaStream_t st);
void launch_repop(const Dims& d, const RepopOp* ops, int nops, const double* oq, double* nq,
                  const double* oqlast, double* nqlast, const double* oqi, double* nqi,
                  const double* oregs, double* nregs, const double* oarea, const double* narea, cudaStream_t st);

// ---- cubed-sphere metric (k_metric.cu) ----------------------------------------
// kind 0: areas from scratch; 1: copy of old slot src[0]; 2: from the four old fine
// slots src[0..3] (igrid order) in cells 0..mx+1, from scratch elsewhere.
struct MetricOp { int kind, dst; int src[4]; };
struct SphereFlow { double axis[3]; double omega; };   // psi = omega (axis . x)
// Areas of every op's patch into narea, then kappa and edge velocities into aux for
// ops of kind 0 and 2.  desc: the new forest's descriptors.
// VTK output: points ((mx+1)(my+1) x 3 doubles) and cell values (mx my x meqn floats)
// of patches order[0..npatch), packed in that order (k_output.cu).
void launch_vtk_pack(const Dims& d, const double* q, const PatchDesc* desc, const int* order, int npatch, int manifold,
                     double* points, float* values, cudaStream_t st);
// ops: the nnew new patches (kind 0 or 2) first, then the nkept kept ones (kind 1)
void launch_sphere_metric(const Dims& d, const MetricOp* ops, int nnew, int nkept, const PatchDesc* desc, int maxlevel,
                          const double* oarea, double* narea, double* aux, const SphereFlow& flow, cudaStream_t st);

}  // namespace fcb
