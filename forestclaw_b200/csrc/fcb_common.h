// fcb_common.h -- plain structs shared by the host driver and the device kernels.
#pragma once
#include <stdint.h>

namespace fcb {

// One leaf patch as seen by the device: physical lower-left corner, mesh widths,
// refinement level and a bit mask of faces on the physical boundary
// (bit f set <=> face f intersects the boundary, fclaw2d_physical_get_bc).
struct PatchDesc {
    double xlower, ylower, dx, dy;
    int level;
    int phys_mask;
    int face_type;      // 2 bits per face: 0 boundary, 1 half (finer nbr), 2 same, 3 double (coarser nbr)
    int flags;          // PATCH_* bits
    int inst;           // instance of a batch of independent forests (0 otherwise)
    int block;          // block of the domain (the cubed sphere's face 0..5; brick tree number)
};

// PATCH_BCC3 << k: corner k of the patch is a corner of the cubed sphere (three blocks meet)
enum { PATCH_HAS_FINE_NBR = 1, PATCH_BCC3 = 2 };

// p*-seed network sizes and layouts (k_mlp.cuh).  The network seeds Newton only
// where the interface carries a wave of strength |dp|/pbar + |du|/cbar above
// MLP_GATE; weaker jumps keep the PVRS start, whose error (below ~1e-2 there) a
// BF16 network does not improve on.
#define MLP_GATE 0.2
enum { MLP_IN = 6, MLP_H = 64, MLP_NPARAM = 64 * 6 + 64 + 64 * 64 + 64 + 64 + 1 };
enum { MLP_OFF_W1 = 0, MLP_OFF_B1 = 384, MLP_OFF_W2 = 448, MLP_OFF_B2 = 4544, MLP_OFF_W3 = 4608, MLP_OFF_B3 = 4672 };
// blob: floats b1 b2 w3 b3 (256 floats), bf16 W1 [64][16] and W2 [64][64] row-major, then
// W1 and W2 again in the tensor cores' K-major core-matrix order (k_tc.cuh kmajor_off)
enum { MLP_BLOB_F_B1 = 0, MLP_BLOB_F_B2 = 64, MLP_BLOB_F_W3 = 128, MLP_BLOB_F_B3 = 192,
       MLP_BLOB_W1_BYTE = 1024, MLP_BLOB_W2_BYTE = 1024 + 64 * 16 * 2, MLP_BLOB_TC_BYTE = 1024 + 64 * 16 * 2 + 64 * 64 * 2,
       MLP_BLOB_TC_LEN = 64 * 16 * 2 + 64 * 64 * 2, MLP_BLOB_BYTES = MLP_BLOB_TC_BYTE + MLP_BLOB_TC_LEN };

// Parameters of one level update launch (clawpack46 method flags and the
// per-step scalars the reference passes through common blocks).
// The levels of one update launch: nlev consecutive levels (1: every patch takes
// the first parameter block), start[k] = first patch of the k-th level (ascending)
// relative to the launch's first patch.
struct LevelGroup {
    int nlev;
    int start[34];
};

struct StepParams {
    int order1, order2;     // method(2), method(3)
    int mthlim[8];
    int mcapa;
    int store_flux;         // time_sync && flux_correction   (clawpack46_time_sync_store_flux)
    int accumulate_waves;   // time_sync && fluctuation_correction (clawpack46_time_sync_accumulate_waves)
    int save_last;          // fclaw2d_clawpatch_save_current_step (q -> qlast)
    int app;                // b4step2 hook
    int wall_faces;         // bit f: mthbc(f) == 3 (reflecting wall)
    double dt;
    double t;
    double grav;
    double dry_tolerance;
    double vt;              // swirl: cos(2 pi (t + dt/2) / T), computed on the host
    double gamma;           // Euler: ratio of specific heats
    double newton_tol;      // Euler: Newton tolerance on the relative change of p*
    unsigned long long* newton_hist;   // Euler: 32-bin histogram of Newton iterations (or null)
    const void* mlp;        // Euler: p*-seed network blob (null: PVRS start)
    const double* inst_dt;  // batch: coarse time step of each instance, dt = this[inst] * (level factor in dt)
    unsigned int* status;   // device status word: STATUS_* bits or'ed in by the kernels (or null)
    // Time-sync registers reset since this level's last update, by face type (bit t for
    // face type t: 0 boundary, 1 half, 2 same, 3 double): the update's first
    // accumulation into such a face's registers starts from zero instead of reading them.
    int reg_reset;
};

// Kernel-side failures reported through the status word (read by the host after a step).
enum { STATUS_NEWTON = 1,       // exact Euler: Newton did not converge from the seed nor from PVRS
       STATUS_DEPTH = 2,        // shallow water: negative depth in a patch
       STATUS_NONFINITE = 4,    // a non-finite value in q
       STATUS_STAGING = 8,      // a patch's asynchronous copy into shared memory did not arrive
       STATUS_TENSOR = 16 };    // a tensor-core MMA of the batched network evaluation did not complete

}  // namespace fcb
