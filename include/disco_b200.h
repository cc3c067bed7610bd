/*
 * disco_b200.h — C-ABI of the B200 (sm_100a) displacement backend for DISCO.
 *
 * Every entry point takes plain pointers and sizes and returns a status code
 * (DISCO_OK on success); no C++ or torch type crosses this boundary.  The C++
 * shim `backend_shim.cpp` re-exposes the four GPU functions of the reference's
 * backend interface (Code/backend.hpp:57-62) on top of these calls, so the
 * reference driver (Code/main.cpp:713-730) selects this backend unchanged.
 *
 * Conventions taken from the reference:
 *   - atoms are SoA doubles, displacements are ACCUMULATED (+=) into arrays
 *     the caller zeroed (Code/backend.hpp:28, Code/backend_cpu.cpp:57-59);
 *   - a line loop's Burgers vector is (phys.bx*mx, phys.by*my, phys.bz*mz)
 *     (Code/backend_cpu.cpp:44-45);
 *   - the box is orthorhombic with lengths box[0..2]; image (i, j, k) moves the
 *     atom by -(i*box[0], j*box[1], k*box[2]) (Code/backend_cpu.cpp:51-54).
 * Errors are status codes; disco_b200_last_error() gives the message.  The
 * reference prints and exits instead (Code/backend_cuda.cu:45-53); the shim
 * maps a non-zero status to exactly that.
 */
#ifndef DISCO_B200_H
#define DISCO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
#define DISCO_OK        0
#define DISCO_EINVAL    1   /* bad argument: null pointer, negative size, bad loop  */
#define DISCO_ENODEV    2   /* no CUDA device usable by this process               */
#define DISCO_ECUDA     3   /* a CUDA runtime call or a kernel launch failed       */
#define DISCO_ENOMEM    4   /* a device or pinned-host allocation failed           */
#define DISCO_ELIMIT    5   /* a size is above a compiled-in or caller capacity    */
#define DISCO_ETIMEOUT  6   /* a bounded device-side wait gave up                  */
#define DISCO_EPLANES   7   /* |b.n| is not a whole number of plane spacings
                               (the reference aborts: Code/prismatic.cpp:50-56)   */

/* ---- precision of the displacement sum ------------------------------------- */
#define DISCO_FP64      0   /* plain drop-in: FP64 throughout                      */
#define DISCO_FP32C     1   /* FP32 bulk on loop-centred coordinates, compensated
                               sums over images and loops, FP64 image offsets     */

/* ---- loop shapes (Code/loop.hpp:13) ----------------------------------------- */
#define DISCO_SHAPE_CIRCLE         0
#define DISCO_SHAPE_RECTANGLE      1
#define DISCO_SHAPE_PARALLELOGRAM  2
#define DISCO_SHAPE_POLYGON        3
#define DISCO_MAX_POLY            32   /* polygon vertices per slab loop            */

/* ---- matter type of a slab loop (Code/prismatic.hpp:40) -------------------- */
#define DISCO_MATTER_NONE          0
#define DISCO_MATTER_VACANCY       1
#define DISCO_MATTER_INTERSTITIAL  2

/* Atom positions (read) and displacements (accumulated).  Code/backend.hpp:29-33.
 * Host pointers for disco_b200_displace, device pointers for
 * disco_b200_plan_execute. */
typedef struct {
    const double *x, *y, *z;
    double *ux, *uy, *uz;
    int64_t n;
} disco_atoms;

/* Loop physics, field for field the reference's LoopPhys (Code/kroupa.hpp:28-36):
 * b = |b| per axis, m and n unit vectors, dS the loopon area. */
typedef struct {
    double bx, by, bz;
    double mx, my, mz;
    double nx, ny, nz;
    double dS;
} disco_loop_phys;

/* One loop as the backend sees it: Code/backend.hpp:20-26 (LoopData).
 * line != 0: closed polyline vx/vy/vz[0..n_vertices-1] (counter-clockwise about
 * n, last vertex joined to the first) with fan apex (cx, cy, cz);
 * line == 0: loopon positions x/y/z[0..n_loopons-1].  Host pointers. */
typedef struct {
    const double *x, *y, *z;
    int32_t n_loopons;
    int32_t line;
    disco_loop_phys phys;
    const double *vx, *vy, *vz;
    int32_t n_vertices;
    int32_t reserved;
    double cx, cy, cz;
} disco_loop;

/* Options of the displacement sum.  The reference's GpuOptions
 * (Code/backend.hpp:53-56) holds fp32 and chunkPairs; images and nu are fixed
 * there at 1 and 0.35 (Code/backend_cpu.cpp:51-53, Code/kroupa.hpp:24) and are
 * parameters here.  Fill with disco_b200_options_default() first. */
typedef struct {
    int32_t precision;     /* DISCO_FP64 or DISCO_FP32C                            */
    int32_t images;        /* image range: -images..+images per axis, 0..8         */
    double  nu;            /* Poisson ratio, in (-1, 0.5)                          */
    double  chunk_pairs;   /* accepted for GpuOptions compatibility; B200 needs no
                              watchdog chunking, so it is ignored                  */
    int32_t atoms_per_thread;  /* 0 = automatic                                    */
    int32_t threads_per_block; /* 0 = automatic                                    */
    int32_t image_split;       /* lanes sharing one atom's images (1..32, power of
                                  two); 0 = automatic                              */
    int32_t verbose;           /* print the reference's per-loop banner lines      */
    double  near_plane;        /* DISCO_FP32C line method: an (atom, loop image)
                                  within near_plane A of the loop plane and within
                                  near_rim A beyond the loop's largest vertex radius
                                  is evaluated in FP64; 0 = defaults (3 A, 3 A)   */
    double  near_rim;
    int32_t stage_kb;          /* shared-memory stage of the streamed tables, KB;
                                  0 = automatic (resident up to 110 KB, else 48)  */
    int32_t image_min;         /* skip the images with max(|i|,|j|,|k|) < image_min:
                                  2 sums only the far shells 2 <= max|n| <= images */
    int32_t stages;            /* batched form: table stages in flight per CTA (the
                                  copy pipeline's depth), 2..4; 0 = 2             */
    int32_t reserved;
} disco_options;

/* Phase timings, seconds: Code/backend.hpp:36-39 (BackendTiming).
 * loop_sec: caller array of nloops entries, or NULL.  All loops run in one
 * launch here, so loop_sec[l] is the kernel time apportioned by loop l's share
 * of the evaluations (never zero for a non-empty loop, as the reference's
 * pair-rate report divides by it: Code/main.cpp:962). */
typedef struct {
    double upload, kernels, download;
    double *loop_sec;
} disco_timing;

/* Work counts of a plan. */
typedef struct {
    int64_t n_loops, n_line_loops, n_loopon_loops;
    int64_t n_segments, n_loopons, n_images;
    double  evals_per_atom;   /* (segments + loopons) x images                     */
} disco_plan_stats;

typedef struct disco_plan disco_plan;

/* ---- device queries ---------------------------------------------------------- */

/* 1 if a CUDA device is usable; replaces gpuAvailable() (Code/backend.hpp:58). */
int disco_b200_available(void);

/* Writes the "--- GPU: <name> ---" banner of printGpuInfo() (Code/backend.hpp:59,
 * Code/backend_cuda.cu:543-553) into buf.  DISCO_ENODEV without a device. */
int disco_b200_device_info(char *buf, size_t len);

/* 1: this build has the FP64 line kernel; replaces gpuLineFp64()
 * (Code/backend.hpp:60).  Always 1 on sm_100a. */
int disco_b200_line_fp64(void);

void disco_b200_options_default(disco_options *opt);

/* Message of the last failing call on this thread (empty if none). */
const char *disco_b200_last_error(void);
const char *disco_b200_strerror(int status);

/* ---- displacement sum ---------------------------------------------------------- */

/* Host buffers in, host buffers out: uploads the atoms, sums every loop over
 * every image in one launch, adds the result into atoms->ux/uy/uz.  Replaces
 * kroupaGPU (Code/backend.hpp:61-62, Code/backend_cuda.cu:568-722). */
int disco_b200_displace(const disco_atoms *atoms, const disco_loop *loops, int32_t nloops,
                        const double box[3], const disco_options *opt, disco_timing *timing);

/* Resident form: the loop tables are built and uploaded once by plan_create;
 * plan_execute adds the field of every loop into DEVICE arrays on `stream`
 * (a cudaStream_t, NULL = legacy default stream) without any host copy. */
int disco_b200_plan_create(const disco_loop *loops, int32_t nloops, const double box[3],
                           const disco_options *opt, int64_t max_atoms, disco_plan **out);
int disco_b200_plan_execute(disco_plan *plan, const disco_atoms *device_atoms, void *stream);
int disco_b200_plan_stats(const disco_plan *plan, disco_plan_stats *stats);
/* Waits for `stream` and reports what the plan's kernels recorded on the
 * device since the last call (DISCO_ETIMEOUT if a bounded wait gave up). */
int disco_b200_plan_sync(disco_plan *plan, void *stream);
int disco_b200_plan_destroy(disco_plan *plan);

/* ---- batched form: many independent samples in one persistent launch ------------ */

/* One sample: its atoms (host pointers for disco_b200_batch, device pointers
 * for disco_b200_batch_plan_create), its loops (host), box and image range.
 * nu and the precision are the batch's (disco_options). */
typedef struct {
    disco_atoms atoms;
    const disco_loop *loops;
    int32_t nloops;
    int32_t images;
    double box[3];
    int32_t image_min;        /* as disco_options.image_min, per sample */
    int32_t reserved;
} disco_sample;

typedef struct disco_batch_plan disco_batch_plan;

/* Batched form of disco_b200_displace: every sample's
 * field is added into its own u.  All samples run in one persistent launch per
 * loop kind over a queue of (sample, atom tile, table chunk) units, balanced
 * across the CTAs by their exact cost; opt->image_split and opt->stage_kb are
 * the tuning knobs (0 = automatic). */
int disco_b200_batch(const disco_sample *samples, int32_t nsamples, const disco_options *opt,
                     disco_timing *timing);

/* Resident form: tables, unit queue and a CUDA graph of the launches are built
 * once; execute replays the graph on `stream` (device atoms given at create). */
int disco_b200_batch_plan_create(const disco_sample *samples, int32_t nsamples,
                                 const disco_options *opt, disco_batch_plan **out);
int disco_b200_batch_plan_execute(disco_batch_plan *plan, void *stream);
int disco_b200_batch_plan_sync(disco_batch_plan *plan, void *stream);
int disco_b200_batch_plan_stats(const disco_batch_plan *plan, disco_plan_stats *stats);
int disco_b200_batch_plan_destroy(disco_batch_plan *plan);

/* ---- learned far-image surrogate: the network ---------------------------------------
 * The reference has no learned path; this is the network of the learned form
 * (14 -> 128 -> 128 -> 128 -> 3, SiLU, BF16 weights and activations on the
 * tensor cores, FP32 accumulation), trained and evaluated by this library's
 * own tcgen05 kernels.  Features are padded to 16 columns and outputs to 16
 * (X: n x 16, Y: n x 16, T: n x 3, all FP32 row-major DEVICE arrays).
 * Parameters: W1[128x16] b1[128] W2[128x128] b2 W3[128x128] b3 W4[16x128] b4[16]
 * as one FP32 vector of disco_b200_mlp_param_count() values. */
typedef struct disco_mlp disco_mlp;

int disco_b200_mlp_create(uint64_t seed, disco_mlp **out);
int disco_b200_mlp_destroy(disco_mlp *m);
int disco_b200_mlp_param_count(void);
int disco_b200_mlp_get_params(const disco_mlp *m, float *host);
int disco_b200_mlp_set_params(disco_mlp *m, const float *host);
int disco_b200_mlp_get_grads(const disco_mlp *m, float *host);
int disco_b200_mlp_forward(disco_mlp *m, const float *X, int64_t n, float *Y, void *stream);
/* forward + backward of the mean squared error over n rows; gradients
 * accumulate in the model until disco_b200_mlp_adam applies and clears them */
int disco_b200_mlp_grad(disco_mlp *m, const float *X, const float *T, int64_t n, float *loss,
                        void *stream);
int disco_b200_mlp_adam(disco_mlp *m, float lr, float beta1, float beta2, float eps,
                        float weight_decay, void *stream);
/* waits for the device and reports a bounded wait of an MLP kernel that gave up */
int disco_b200_mlp_status(disco_mlp *m);

/* ---- learned far-image surrogate: features, inference, learned displacement ----------
 * The network stands in for a line loop's field summed over the far image shells
 * image_min <= max(|i|,|j|,|k|) <= images.  Its 14 features for atom r and loop
 * (centre c, area A, largest vertex radius rho_max, unit normal n, Burgers vector b;
 * box L = (Lx, Ly, Lz), Lref = (Lx Ly Lz)^(1/3)):
 *     0-2  (r-c)_x / Lx, (r-c)_y / Ly, (r-c)_z / Lz   position relative to the loop
 *          centre over the box lengths (loop-centred frame, box axes, in (-1, 1))
 *     3    sqrt(A / pi) / Lref          loop radius over box edge
 *     4-6  n                            plane normal
 *     7-9  b / |b|                      Burgers vector direction
 *     10   Ly / Lx - 1, 11 Lz / Lx - 1  box aspect ratios
 *     12   rho_max / sqrt(A / pi) - 1   shape (0 for a circle)
 *     13   (b / |b|) . n                0 for a glide loop
 * each entering as (raw - mu) * inv_sd (features 14, 15 are zero padding).  The
 * network's outputs 0-2 times gain = out_scale |b| A / Lref^2 are the loop's
 * displacement (A, box axes) summed over those shells. */
typedef struct {
    float mu[16];
    float inv_sd[16];
    float out_scale;
    int32_t images;           /* the shells the network was trained for */
    int32_t image_min;
    int32_t reserved;
} disco_far_norm;

/* Features of every (loop, atom) pair, loop-major: X[(l n + i) 16 + k] (DEVICE,
 * FP32).  norm NULL: raw features (mu 0, inv_sd 1) and gain without out_scale.
 * gain: DEVICE array of nloops floats, or NULL.  Line loops only. */
int disco_b200_far_features(const disco_atoms *device_atoms, const disco_loop *loops, int32_t nloops,
                            const double box[3], const disco_far_norm *norm, float *X, float *gain,
                            void *stream);

/* The network's far-shell displacement of the loops loop_sel[0..nsel) (host
 * indices; NULL = all nloops) at every atom, in one fused tcgen05 kernel:
 * features, four layers and the gain.  per_loop NULL: added into the atoms'
 * ux/uy/uz; else written to per_loop[(j 3 + c) n + i] (DEVICE, FP32) for the
 * j-th selected loop.  One call at a time per network. */
int disco_b200_far_apply(disco_mlp *m, const disco_far_norm *norm, const disco_atoms *device_atoms,
                         const disco_loop *loops, int32_t nloops, const double box[3],
                         const int32_t *loop_sel, int32_t nsel, float *per_loop, void *stream);

typedef struct {
    int32_t precision;        /* near shell and fallback loops: DISCO_FP32C or DISCO_FP64 */
    int32_t check_precision;  /* exact far shells on the check subsample              */
    double  nu;
    double  check_fraction;   /* share of the atoms re-checked every call (0.01)      */
    double  tol_loop;         /* a loop whose network error exceeds this on the
                                 subsample is summed exactly (1e-3 A)                */
    double  tol_total;        /* further loops fall back, largest error first, until
                                 the subsample's total far-shell error is within this */
    uint64_t seed;            /* subsample: one atom drawn in each of n_check equal
                                 index strata                                        */
} disco_learned_options;

typedef struct {
    int64_t n_check;          /* atoms in the check subsample                          */
    int32_t n_fallback;       /* loops whose far shells were summed exactly            */
    int32_t launches;         /* kernels this call launched                            */
    double  check_max;        /* max |du| of the network's part on the subsample, A   */
    double  check_rms;
    double  worst_loop;       /* largest per-loop max |du| before any fallback, A      */
    double  t_check, t_near, t_far, t_fallback;   /* device seconds of each phase      */
    double *loop_err;         /* caller array of nloops or NULL: per-loop max |du|     */
    int32_t *fallback;        /* caller array of nloops or NULL: 1 = summed exactly    */
} disco_learned_report;

/* Learned displacement: u += the exact field of every loop over the near images
 * max|n| < norm->image_min (opt->precision) plus the network's far shells
 * image_min <= max|n| <= norm->images, with the exact far-shell sum
 * (opt->check_precision: DISCO_FP64, or DISCO_FP32C, within about 1e-5 A of
 * FP64 on a whole sum and twice as fast) recomputed per loop on a random atom
 * subsample every call and replacing the network for the loops that miss the
 * tolerances.
 * DEVICE atoms; the call returns when the work is done. */
int disco_b200_learned_displace(disco_mlp *m, const disco_far_norm *norm, const disco_atoms *device_atoms,
                                const disco_loop *loops, int32_t nloops, const double box[3],
                                const disco_learned_options *opt, disco_learned_report *report,
                                void *stream);

/* ---- input on the device ------------------------------------------------------------ */

/* Perfect-lattice sites written straight into DEVICE arrays x, y, z of
 * 2 (BCC, lattice 0) or 4 (FCC, lattice 1) x nx x ny x nz entries:
 * Code/lattice.hpp:35-51 (generateLattice), same order, bit-identical
 * positions, without the host build and the host-to-device copy.  Runs on
 * `stream` and returns without waiting. */
int disco_b200_lattice(int32_t lattice, int32_t nx, int32_t ny, int32_t nz, double a0,
                       double *x, double *y, double *z, void *stream);

/* ---- output ------------------------------------------------------------------------- */

/* The atom lines of the output files, formatted on the device as the
 * reference's C++ streams format them (`fixed << setprecision(8)`: exact
 * decimal rounding, ties to even).  format 0: XYZ, "<element> x y z\n"
 * (Code/main.cpp:826-831); format 1: LAMMPS atomic, "<k+1> 1 x y z\n"
 * (Code/main.cpp:86-92) for an orthorhombic box, whose projection onto the
 * LAMMPS frame is the identity.  x, y, z: DEVICE arrays of final positions
 * (e.g. from disco_b200_finalize_resident), |v| < 1.8e11; out: DEVICE buffer of
 * `capacity` bytes; *bytes = the text's length.  A short buffer returns
 * DISCO_ELIMIT with *bytes = the size needed.  The call waits for the line
 * lengths, then launches the writing kernel on `stream` and returns.  The
 * header lines stay with the caller (they hold a handful of numbers). */
int disco_b200_format_atoms(int32_t format, const char *element, const double *x, const double *y,
                            const double *z, int64_t n, char *out, int64_t capacity, int64_t *bytes,
                            void *stream);

/* ---- self-test ---------------------------------------------------------------------- */

/* Evaluates one of the kernels' own FP64 routines on DEVICE arrays, so that
 * tests can hold them against CUDA's functions: fn 0: 1/sqrt(x) (hardware
 * approximation + one Householder step), 1: 1/x (approximation + one cubic
 * Newton-Raphson step), 2, 3, 4: 2 atanh(x) by the 8-, 6- and 4-term series
 * of the far-field J0.  No counterpart in the reference. */
int disco_b200_math_check(int32_t fn, const double *x, double *y, int64_t n, void *stream);

/* ---- prismatic loops: slab selection and stream compaction ------------------------ */

/* One loop of the matter step.  Geometry as in the reference's loop class
 * (Code/loop.hpp:19-45): centre c on a mid-plane, unit m and n, |b| = bmag,
 * in-plane grid axes u, v (oblique for a parallelogram), shape parameters, and
 * for a polygon the vertex, inner-vertex and inward-normal arrays (pu..nv). */
typedef struct {
    double c[3], m[3], n[3];
    double bmag;
    double u[3], v[3];
    double spacing;             /* d: atomic-plane spacing of the n family            */
    int32_t shape;              /* DISCO_SHAPE_*                                       */
    int32_t n_poly;             /* polygon vertex count, <= DISCO_MAX_POLY             */
    double radius, half_m, half_p, r_corner;
    double pu[DISCO_MAX_POLY], pv[DISCO_MAX_POLY];
    double qu[DISCO_MAX_POLY], qv[DISCO_MAX_POLY];
    double nu[DISCO_MAX_POLY], nv[DISCO_MAX_POLY];
    double shift_pos[3];        /* copy shift of a side +1 atom (interstitial): +b,
                                   plus the Shockley shift of a Frank loop
                                   (Code/main.cpp:630-650)                           */
    double shift_neg[3];        /* copy shift of a side -1 atom                        */
    int32_t apply;              /* 0: "Matter: none", displacement only (main.cpp:593) */
    int32_t reserved;
} disco_slab_loop;

/* Per-loop result, the scalar part of SlabResult (Code/prismatic.hpp:47-55). */
typedef struct {
    int32_t type;               /* DISCO_MATTER_*                                      */
    int32_t planes;             /* k                                                   */
    double  height, spacing;    /* |b.n|, d                                            */
    double  b[3];               /* |b| m                                               */
    int64_t offset, count;      /* this loop's entries in slab_atoms / slab_side       */
} disco_slab_info;

/* An interstitial copy after compaction: source atom (new index) and shift. */
typedef struct {
    int32_t atom;
    int32_t reserved;
    double  shift[3];
} disco_copy;

/* Matter step of Code/main.cpp:586-687 on the GPU, host buffers.
 * For every loop with b.n != 0 and apply != 0: the slab atoms of prismaticSlab
 * (Code/prismatic.cpp:36-74), ascending, with their side; vacancy slabs are
 * removed and interstitial slabs give copies (loop order, then slab order).
 * Outputs: survivors x_out/y_out/z_out[0..counts[0]) in original order,
 * new_index[n] (-1 for a removed atom), info[nloops], slab_atoms/slab_side
 * (capacity slab_capacity, entries of loop l at info[l].offset), copies
 * (capacity copy_capacity) with their source renumbered and copies of removed
 * atoms dropped.  counts = {survivors, slab entries, copies}; when a capacity
 * is too small the call returns DISCO_ELIMIT with counts holding the sizes
 * needed.  Selection is bit-exact with the reference's FP64 predicate.  On the
 * device: one cooperative kernel (each atom's slab mask computed once, counts
 * per CTA, grid barriers around a scan of those counts, then the ordered
 * writes of survivors, slab entries and copies).  Output arrays must not
 * overlap the inputs. */
int disco_b200_prismatic(const double *x, const double *y, const double *z, int64_t n,
                         const disco_slab_loop *loops, int32_t nloops, const double box[3],
                         double *x_out, double *y_out, double *z_out, int32_t *new_index,
                         disco_slab_info *info,
                         int32_t *slab_atoms, int8_t *slab_side, int64_t slab_capacity,
                         disco_copy *copies, int64_t copy_capacity,
                         int64_t counts[3]);

/* The matter step above for callers that cannot let this library allocate
 * device memory (their own allocator owns the GPU, or cudaMalloc/cudaFree and
 * the device synchronisation they imply are not allowed where they call).
 * No counterpart in the reference.  Inputs x, y, z and every output array
 * except info and counts are DEVICE pointers the caller allocated; loops,
 * box, info and counts are host memory.  Work is queued on `stream` (a
 * cudaStream_t; NULL = legacy default stream) and the call waits for it once,
 * at the end, to read the totals.  Scratch lives in a fixed 8 MiB device
 * array inside the library (held by every GPU that loads it until the process
 * exits): at most 16 777 216 atoms, 64 prismatic loops and 65 536 atoms in
 * slabs per call, DISCO_ELIMIT beyond.  The first call on a device looks up
 * that array's device address (again after a device reset gives the device a
 * new context), so make it before any stream capture.  All calls share the
 * array: calls whose work overlaps on the GPU (other streams, other host
 * threads on the same device) race and must be serialised by the caller.
 * Capacities: slab entries beyond slab_capacity and copies beyond
 * copy_capacity are not written, and the call returns DISCO_ELIMIT with
 * counts[1] and counts[2] holding the sizes needed.  The device outputs match
 * disco_b200_prismatic's bit for bit. */
int disco_b200_prismatic_noalloc(const double *x, const double *y, const double *z, int64_t n,
                                 const disco_slab_loop *loops, int32_t nloops, const double box[3],
                                 double *x_out, double *y_out, double *z_out, int32_t *new_index,
                                 disco_slab_info *info,
                                 int32_t *slab_atoms, int8_t *slab_side, int64_t slab_capacity,
                                 disco_copy *copies, int64_t copy_capacity,
                                 int64_t counts[3], void *stream);

/* Code/main.cpp:733-743 and 797-818 fused: appends the copies (position of the
 * source, displacement u(source) + shift) after the n atoms, then writes the
 * wrapped final positions r = x + u, folded once into [-L/2, L/2] and shifted
 * by +L/2.  Output arrays hold n + ncopies entries; ux/uy/uz_out may be NULL. */
int disco_b200_finalize(const double *x, const double *y, const double *z,
                        const double *ux, const double *uy, const double *uz, int64_t n,
                        const disco_copy *copies, int64_t ncopies, const double box[3],
                        double *fx, double *fy, double *fz,
                        double *ux_out, double *uy_out, double *uz_out);

/* Resident form of disco_b200_finalize: every array, copies included, is a
 * DEVICE pointer (copies as written by disco_b200_prismatic_noalloc); the
 * kernel runs on `stream` and the call returns without waiting.  Copy sources
 * must lie in [0, n) (they do when they come from the matter step). */
int disco_b200_finalize_resident(const double *x, const double *y, const double *z,
                                 const double *ux, const double *uy, const double *uz, int64_t n,
                                 const disco_copy *copies, int64_t ncopies, const double box[3],
                                 double *fx, double *fy, double *fz,
                                 double *ux_out, double *uy_out, double *uz_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DISCO_B200_H */
