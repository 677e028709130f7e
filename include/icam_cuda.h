/*
 * icam_cuda.h — the C ABI of the B200 exact part field.
 *
 * These entry points replace the reference's GPU host for the part field,
 * `PartGpu` (crates/icam-sim/src/partgpu.rs), and the level bake of its brick
 * cache, `PartCache::level` (crates/icam-sim/src/partcache.rs:433-506). Every
 * argument is a plain pointer or size: the caller owns all host arrays, the
 * library owns the device memory inside an IcamPack. Each pack has its own CUDA
 * stream; calls on one pack must not overlap (serialise them, as the reference
 * serialises its dispatches on one queue).
 *
 * Values follow the reference kernel's contract (crates/icam-core/src/solid3/
 * gpu.wgsl:1909-1921): each node or point comes back as (value, flag) with flag
 * 0 = the exact signed distance, 1 = only a lower bound past the clamp is known
 * (value = that bound, its sign to come from a neighbour), 2 = undecided.
 *
 * The brick layout is the reference's (crates/icam-sweep/src/cache.rs:69-92):
 * 8 x 8 x 8 cells, 9 x 9 x 9 nodes x fastest, each stored as
 * round(clamp(d / clamp, -1, 1) * 32767) in an i16, two to a 32-bit word low half
 * first, 365 words a brick; the map holds a slot or ICAM_AIR / ICAM_SOLID.
 */
#ifndef ICAM_CUDA_H
#define ICAM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "icam_solid.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ICAM_AIR 0xffffffffu   /* cache.rs:84 AIR */
#define ICAM_SOLID 0xfffffffeu /* cache.rs:85 SOLID */
#define ICAM_WORDS 365         /* cache.rs:91 WORDS */
#define ICAM_READ 0xfffffff0u  /* a brick the box decision leaves to be read (icam_decide_level) */
#define ICAM_NODES 729

/* Arithmetic of the per-node evaluation. */
enum {
  ICAM_FP64 = 0,          /* every step in double precision */
  ICAM_MIXED = 1,         /* single-precision bulk, double-precision polish, trim near loops and signs */
  ICAM_MIXED_LEARNED = 2  /* ICAM_MIXED seeded by the pack's trained seed network (a solid with no
                             B-spline sub-patch has nothing to seed: ICAM_MIXED) */
};

/* Status codes. */
enum {
  ICAM_OK = 0,
  ICAM_ERR_ARG = 1,     /* a bad argument (message in err) */
  ICAM_ERR_CUDA = 2,    /* a CUDA call failed */
  ICAM_ERR_PACK = 3,    /* the solid could not be packed */
  ICAM_ERR_ROOM = 7,    /* a device work list overflowed (gpu.wgsl why-code 7) */
  ICAM_ERR_BUDGET = 8   /* a bounded device loop gave up (gpu.wgsl why-code 8) */
};

typedef struct IcamPack IcamPack;

typedef struct IcamPackOptions {
  int device;    /* CUDA device ordinal */
  double need;   /* distance (mm) within which B-spline sub-patches should certify */
} IcamPackOptions;

typedef struct IcamBakeStats {
  int64_t boxes_read;      /* box centres read by the decision */
  int64_t bricks_read;     /* bricks the decision reads (its boxes of one brick) */
  int64_t bricks_words;    /* of those, bricks stored as words (not air or solid) */
  int64_t nodes_exact;     /* flag 0 nodes */
  int64_t nodes_far;       /* flag 1 nodes, signed by the fill */
  int64_t nodes_undecided; /* flag 2 nodes left after the device fallback (bridged) */
  int64_t pairs;           /* (brick, candidate) pairs evaluated */
  int64_t fallback_nodes;  /* nodes sent to the subdivision fallback */
  int64_t kernel_launches; /* kernels launched by the call */
  double ms_decide, ms_cull, ms_nodes, ms_post; /* device time by stage */
  /* Candidates listed for the bricks read, summed over them, by kind as the
   * reference's census counts them (Exact::near_kinds, solid3.rs:1727): analytic
   * faces, B-spline spans (distinct spans of the sub-patches listed), line or arc
   * edges, spline edge pieces, vertices. */
  int64_t census[5];
  /* Read bricks whose every node lies on one side of the surface by more than an i16
   * step, known from the brick's centre distance (the field is 1-Lipschitz): air or
   * solid without reading their nodes. */
  int64_t bricks_settled;
  /* Bytes the call copied from host to device (the decision's first boxes) and from
   * device to host (its counts, and for icam_bake_level the map and atlas). */
  int64_t h2d_bytes, d2h_bytes;
  /* The mixed forms: nodes the single-precision walk left to the double walk (a
   * distance near zero, a stalled or uncertified solve, a deferred feature). */
  int64_t nodes_double;
  /* The mixed forms: box centres the decision's float reading left to the double walk
   * (a verdict within the float error of its threshold, a value near zero). */
  int64_t centres_double;
  /* The mixed forms' brick kernel: single-precision Newton solves of sub-patches at the
   * nodes, and the patch evaluations they took (the iterations). */
  int64_t newton_solves, newton_evals;
} IcamBakeStats;

/* Packs the solid for the device (PartGpu::new, partgpu.rs:132; Exact::gpu_pack,
 * crates/icam-core/src/solid3/gpu.rs:259). Returns ICAM_OK and *out, or an error
 * with a message in err. A B-spline face's creases (interior knot lines where its
 * normal jumps, Exact::c0_line, solid3.rs:1821-1886) are packed as the face's own
 * edges; a side of a B-spline face's domain collapsed to one point inside the face
 * (a pole, solid3.rs:1615-1625) is packed as a point feature with the fan
 * pseudo-normal (fan_normal, solid3.rs:1960-1986), after the solid's vertices.
 * ICAM_ERR_PACK, before any device work, for a crease that crosses its face's loops or
 * a B-spline face whose normal vanishes off its collapsed sides. */
int icam_pack_create(const IcamSolidDesc* solid, const IcamPackOptions* opt, IcamPack** out, char* err,
                     size_t errlen);

void icam_pack_destroy(IcamPack* pack);

/* Counts of what the pack holds: faces, edges, point features (vertices, then
 * poles), B-spline sub-patches, edge pieces, trim cells, tree nodes. */
int icam_pack_info(const IcamPack* pack, int64_t counts[7]);

/* Signed distance of n points (x, y, z), each (value, flag) as above. With
 * capped != 0 a point needs an exact value only within `clamp` (past it the
 * answer may be the bound, flag 1), as PartGpu::points_scatter_capped
 * (partgpu.rs:249); with capped == 0 every point is read exactly
 * (PartGpu::points_refined, partgpu.rs:243). Host arrays. Points are read in double
 * precision: `precision` must be ICAM_FP64 (the mixed forms, which rebase and seed
 * their float solves per brick, are brick reads), else ICAM_ERR_ARG. */
int icam_points(IcamPack* pack, const double* xyz, size_t n, double clamp, int capped, int precision,
                double* value_out, int8_t* flag_out);

/* The 729 nodes of each brick whose first node is first_nodes[i] (cell side h),
 * exact within `clamp` (PartGpu::bricks / bricks_scatter, partgpu.rs:227-241):
 * values_out n x 729 (value, flag) as float pairs, as the reference returns them;
 * d_out (optional) the same values in double. Candidates are listed on the device
 * (the reference lists them on the CPU, GpuPack::list, gpu.rs:709). */
int icam_bricks(IcamPack* pack, const double* first_nodes, size_t n, double h, double clamp, int precision,
                float* values_out, double* d_out);

/* icam_bricks without allocation. No counterpart in the reference: it is for
 * callers that may not allocate device or host memory during the call (memory
 * reserved up front for the stock model; a loop that cannot take the device-wide
 * wait of cudaFree). Same kernel and outputs as icam_bricks, with every buffer in
 * one fixed device array of the library (one per device, about 3 MB) that all
 * calls on that device share: calls that overlap in time race on it. n above
 * ICAM_STATIC_BRICKS is refused with ICAM_ERR_ROOM; ICAM_MIXED_LEARNED on a pack
 * whose seed network is neither trained nor loaded with ICAM_ERR_ARG, as icam_bricks
 * refuses it. The call is synchronous: it returns once the results are in values_out
 * / d_out (host memory), so it may never be made while a stream of the device is
 * being captured. The first call on a device resolves the array's address and may
 * load the library's device code. The address is kept until the process
 * exits, so no call may follow a cudaDeviceReset of that device. Errors are written
 * to err (errlen bytes), not to the pack's message. */
#define ICAM_STATIC_BRICKS 256
int icam_bricks_static(IcamPack* pack, const double* first_nodes, size_t n, double h, double clamp, int precision,
                       float* values_out, double* d_out, char* err, size_t errlen);

/* One level of the brick cache (PartCache::level, partcache.rs:433): bricks of
 * 8 x 8 x 8 cells of side h, the first node at lo, nb bricks along each axis,
 * the box grid aligned on `origin` (the stock's low corner; partcache.rs:250-259),
 * values clamped to `clamp` (h sqrt(3) in the reference). Decides every brick on
 * the device (partcache.rs:226-331), reads the others' nodes, signs the far nodes,
 * bridges the undecided ones, quantises and packs them (partcache.rs:759-970).
 * map_out: nb[0]*nb[1]*nb[2] entries, x fastest (slot, ICAM_AIR or ICAM_SOLID);
 * atlas_out: up to atlas_cap_words words, slots of 365 words in brick order;
 * *n_slots: the slots written. A NULL atlas_out returns *n_slots only, and an atlas_out
 * too small for them ICAM_ERR_ARG; either way the level stays on the device for
 * icam_level_read, so sizing the atlas needs no second bake. */
int icam_bake_level(IcamPack* pack, double h, const double lo[3], const int64_t nb[3], double clamp,
                    const double origin[3], int precision, uint32_t* map_out, uint32_t* atlas_out,
                    size_t atlas_cap_words, size_t* n_slots, IcamBakeStats* stats);

/* The box decision of a level alone (PartCache::decide, partcache.rs:226-331), with the
 * arguments of icam_bake_level: map_out (nb[0]*nb[1]*nb[2] entries, x fastest) holds
 * ICAM_AIR / ICAM_SOLID for the bricks decided and ICAM_READ for the bricks to read;
 * read_out / dc_out (optional, read_cap entries) the bricks to read in brick order
 * (partcache.rs:486) and their centres' signed distances (NaN where the decision does
 * not need one); *n_read their count (ICAM_ERR_ARG when above read_cap with an output
 * given). stats: boxes_read, bricks_read, kernel_launches, ms_decide. The mixed forms
 * decide the same bricks as ICAM_FP64. */
int icam_decide_level(IcamPack* pack, double h, const double lo[3], const int64_t nb[3], double clamp,
                      const double origin[3], int precision, uint32_t* map_out, int64_t* read_out, double* dc_out,
                      size_t read_cap, size_t* n_read, IcamBakeStats* stats);

/* The last level baked on the pack (by icam_bake_level or icam_bake_level_device),
 * copied out without baking again: map_out (map_entries = the level's
 * nb[0]*nb[1]*nb[2] entries) and atlas_out (atlas_cap_words >= n_slots x 365), either
 * may be NULL. The sizing pattern is one bake with atlas_out NULL for *n_slots, then
 * this read into an atlas of that size. The outputs may be host arrays or device memory
 * (the copy's direction follows from the addresses), so a caller that keeps the level on
 * its GPUs reads it into buffers of its own. No counterpart in the reference, whose level
 * bake returns owned vectors. ICAM_ERR_ARG when no level was baked or a size is wrong. */
int icam_level_read(IcamPack* pack, uint32_t* map_out, size_t map_entries, uint32_t* atlas_out,
                    size_t atlas_cap_words);

/* The same bake, its results left in device memory the pack owns (valid until the
 * next bake on the pack; the pack's point and brick reads do not touch them):
 * *d_map and *d_atlas are device pointers. For callers that consume the level on the
 * GPU (the reference's viewer uploads it to its ray caster). */
int icam_bake_level_device(IcamPack* pack, double h, const double lo[3], const int64_t nb[3], double clamp,
                           const double origin[3], int precision, const uint32_t** d_map,
                           const uint32_t** d_atlas, size_t* n_slots, IcamBakeStats* stats);

/* The candidate features within reach of a point's box, as the device lists them
 * (PartGpu::list, partgpu.rs:220): codes kind << 28 | index (kinds: 0 analytic
 * face, 1 B-spline sub-patch, 2 line or arc edge, 3 spline edge piece, 4 vertex).
 * Host-only, reentrant. */
int icam_list(const IcamPack* pack, const double c[3], double r, double d, uint32_t* codes, size_t cap,
              size_t* n);

/* Keeps the device busy for `secs` so its clocks are up (PartGpu::warm, partgpu.rs:188). */
int icam_warm(IcamPack* pack, double secs);

/* Measures the device's fused multiply-add throughput in double (precision
 * ICAM_FP64) or single (ICAM_MIXED) precision: a kernel of independent FMA chains
 * on every SM, timed with events on the pack's stream. *flops: FLOP/s (2 a FMA).
 * No counterpart in the reference; the roofline denominators of the bench. */
int icam_probe_fma(IcamPack* pack, int precision, double* flops);

/* The CUDA stream (a cudaStream_t) the pack's calls run on, for callers that order
 * their own work or events around them. */
void* icam_pack_stream(const IcamPack* pack);

/* The last error message of a call on this pack. */
const char* icam_last_error(const IcamPack* pack);

/* The solid's box (Exact's tree root, solid3.rs:97-236). */
int icam_pack_box(const IcamPack* pack, double lo[3], double hi[3]);

/* ---- Batches: many parts baked together. No counterpart in the reference, which bakes
 * one part a call (PartCache::level, partcache.rs:433). Each part's box decision runs on
 * its own pack; then every part's read bricks go through one launch of the brick kernel
 * fed by a device work queue, one scan and one assembly, captured as a CUDA graph and
 * replayed while the batch's levels and sizes stay the same. The brick kernel's tiling
 * (warps a block) is picked by timing each choice on the batch's first bake. A part's
 * results are the same as icam_bake_level_device's for that part alone. */
typedef struct IcamBatch IcamBatch;

typedef struct IcamBatchLevel { /* one part's level, as icam_bake_level takes it */
  double h;
  double lo[3];
  int64_t nb[3];
  double clamp;
  double origin[3];
  int32_t has_origin;
  int32_t pad;
} IcamBatchLevel;

typedef struct IcamBatchPart { /* one part's level, in device memory */
  const uint32_t* d_map;       /* nb[0] x nb[1] x nb[2] entries (in the batch) */
  const uint32_t* d_atlas;     /* n_slots x 365 words (in the batch) */
  size_t n_slots;
  int64_t bricks_read;
} IcamBatchPart;

typedef struct IcamBatchStats {
  int64_t parts, boxes_read, bricks_read, bricks_words, nodes_exact, nodes_undecided;
  int64_t kernel_launches;
  int32_t warps;           /* the tiling in use: warps a block of the brick kernel */
  int32_t graph_replayed;  /* 1: the post-decision graph was replayed, 0: captured */
  double tune_ms[3];       /* the tuning's times for 1, 2 and 4 warps a block */
  double ms_decide, ms_bricks;
  int64_t bricks_settled;  /* as IcamBakeStats::bricks_settled */
} IcamBatchStats;

/* A batch over n packs on one device (a pack may appear more than once, e.g. to bake one
 * part at two resolutions). The packs must outlive it; a pack's own calls and a batch
 * bake that uses it must not run at the same time. */
int icam_batch_create(IcamPack* const* packs, size_t n, IcamBatch** out, char* err, size_t errlen);
void icam_batch_destroy(IcamBatch* batch);
/* Bakes levels[i] of part i, all parts together; parts_out[i] its results, valid until
 * the next bake of the batch. */
int icam_batch_bake(IcamBatch* batch, const IcamBatchLevel* levels, int precision, IcamBatchPart* parts_out,
                    IcamBatchStats* stats);
const char* icam_batch_last_error(const IcamBatch* batch);
/* A part's map (map_entries of them) and atlas (atlas_cap_words >= its n_slots x 365)
 * copied to host arrays. */
int icam_batch_read(IcamBatch* batch, const IcamBatchPart* part, size_t map_entries, uint32_t* map_out,
                    uint32_t* atlas_out, size_t atlas_cap_words);

/* ---- The seed network (ICAM_MIXED_LEARNED). No counterpart in the reference, which
 * starts every Newton solve on a B-spline sub-patch at its centre: a small MLP
 * (query in the sub-patch's frame + a 16-number descriptor -> 64 -> 64 -> 64 ->
 * (s, t, distance / L)) predicts the start; each start is checked by the solve it
 * starts (convergence and the critical-point test), with the centre start as the
 * fallback, so the answers stay the exact evaluator's. Trained on the device by the
 * library's own kernels on pairs the exact FP64 evaluator makes; run on the tensor
 * cores in BF16. Weights live in the pack; the parameter vector's layout is
 * W1[32][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64][8] b4[8] (row = input,
 * column = output; inputs past 19 and outputs past 3 are padding). */

/* n training pairs from the exact evaluator (sub-patch points moved along the normal
 * by up to `need` and across the patch): x_out n x 32 inputs (19 used), y_out n x 4
 * targets (s, t, d / L, 1). */
int icam_seednet_samples(IcamPack* pack, size_t n, uint64_t seed, double need, float* x_out, float* y_out);

/* Reads (get) and/or sets (set) the FP32 parameters; *n_params their count. */
int icam_seednet_params(IcamPack* pack, float* get, const float* set, size_t* n_params);

/* The gradient of the mean loss (s - s*)^2 + (t - t*)^2 + 0.1 (d - d*)^2 over the n
 * pairs (x n x 32, y n x 4) at the current parameters, and that loss. */
int icam_seednet_grad(IcamPack* pack, const float* x, const float* y, size_t n, float* grad_out, double* loss_out);

/* Trains for `steps` Adam steps of `batch` fresh pairs each (one CUDA graph replayed);
 * loss_out (optional, steps floats) the loss of every step. */
int icam_seednet_train(IcamPack* pack, int64_t steps, int64_t batch, uint64_t seed, double need, double lr,
                       float* loss_out);

/* The net's starts against the centre start on n fresh pairs: stats[0] pairs, [1] mean
 * Newton iterations from the net, [2] from the centre, [3] and [4] their 99th
 * percentiles, [5] the fallback rate, [6] pairs whose answers differ by more than
 * 1e-9 of the sub-patch's size, [7] the largest such difference over that size. */
int icam_seednet_ab(IcamPack* pack, size_t n, uint64_t seed, double need, double stats[8]);

#ifdef __cplusplus
}
#endif

#endif /* ICAM_CUDA_H */
