/* bhg.h - C ABI of the B200 Barnes-Hut hot path.
 *
 * A drop-in for the grouped pass of the reference solver
 * (devreal/AMT-BH-benchmark, ttg-parsec/src).  In the reference, one force
 * evaluation is two C++ calls inside step_particles' grouped branch
 * (integrate_ttg.h:88-107):
 *
 *   build_flat_tree(FlatTree&, BuildScratch&, particles, max_leaf, group_size)
 *                                                   flat_build_ttg.h:276-281
 *   run_grouped_pass(FlatTree&, ForceParams, target_size, on_result)
 *                                                   grouped_ttg.h:297-323
 *
 * followed by the kick/drift callback (integrate_ttg.h:74-77) and the swap
 * of the caller's particle vector with the Morton-ordered one (:107).  This
 * ABI keeps those phase boundaries - build the tree, compute multipoles,
 * walk forces, integrate - over a particle array that stays resident in
 * GPU memory between calls.  All entry points return 0 on success or a
 * BHG_E* code; bhg_last_error() gives the message.  No C++ exception crosses
 * the ABI.  A context owns one CUDA stream; its calls are asynchronous except
 * where stated (download, status queries).  One context per host thread.
 */
#ifndef BHG_H
#define BHG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes. */
#define BHG_OK 0
#define BHG_EINVAL 1      /* bad argument */
#define BHG_ECUDA 2       /* a CUDA call failed */
#define BHG_ENOMEM 3      /* the HBM budget or the device ran out */
#define BHG_ENONFINITE 4  /* a particle coordinate is NaN or infinite */
#define BHG_ESTATE 5      /* call out of order (e.g. walk before build) */
#define BHG_EDEVICE 6     /* a kernel reported an internal limit (see message) */
#define BHG_ECANCELLED 7  /* serving: the request was cancelled */
#define BHG_EAGAIN 8      /* bhg_sync: not every enqueued evaluation ran (see message); run them again */

/* bh::Particle (particle.h:7-24): 64 bytes, 4 bytes of padding after id. */
typedef struct bh_particle64 {
  uint32_t id;
  uint32_t pad;
  double mass;
  double pos[3];
  double vel[3];
} bh_particle64;

typedef struct bhg_context bhg_context;

typedef struct bhg_config {
  int device;           /* CUDA device ordinal */
  uint64_t hbm_budget;  /* bytes this context may allocate; 0 = no limit */
  uint32_t flags;       /* reserved, 0 */
} bhg_config;

/* Walk arithmetic. */
#define BHG_PRECISION_SPLIT 0 /* FP32 offsets from the target centre, FP64 sums */
#define BHG_PRECISION_FP64 1  /* all-FP64 walk (the plain path) */

/* ForceParams (traversal_ttg.h:136-141) plus the walk's arithmetic. */
typedef struct bhg_force_params {
  double theta;
  double eps2;
  double G;
  int use_quadrupole;
  int precision;
} bhg_force_params;

/* Device time per phase, summed over the evaluations since the last reset
 * (CUDA events recorded around each phase on the context's stream), and the
 * interaction counts of those evaluations. */
typedef struct bhg_stats {
  double pre_ms;       /* bounds, domain, Morton keys, digit histograms */
  double sort_ms;      /* the radix-sort passes */
  double tree_ms;      /* gather into Morton order + octree topology */
  double multipole_ms; /* upward pass */
  double targets_ms;   /* walk targets */
  double walk_ms;      /* force walk with fused kick/drift */
  double last_walk_ms; /* the most recent walk alone */
  uint64_t pp;         /* particle-particle interactions (monopole cells included in no-quad mode) */
  uint64_t pc;         /* particle-cell quadrupole interactions */
  uint32_t evals;      /* walks timed */
  uint32_t nodes;      /* octree nodes of the last build */
  uint32_t targets;    /* walk targets of the last walk */
  uint32_t depth;      /* levels of the last build */
  uint32_t sort_passes;
  uint32_t kernels_per_eval; /* kernel launches of one evaluation (bhg_step) */
} bhg_stats;

/* ---- lifetime ---------------------------------------------------------- */

/* Replaces GroupedWorkspace (integrate_ttg.h:61-64): storage reused across
 * steps, grown and never shrunk. */
int bhg_create(bhg_context** ctx, const bhg_config* cfg);
int bhg_destroy(bhg_context* ctx);
const char* bhg_last_error(const bhg_context* ctx);
/* Run this context's work on a caller-owned cudaStream_t (NULL: its own). */
int bhg_set_stream(bhg_context* ctx, void* cuda_stream);

/* ---- particles ----------------------------------------------------------- */

/* Copies n particles (bh::Particle layout) from host memory into the context
 * as one system.  Replaces handing the particle vector to build_flat_tree
 * (flat_build_ttg.h:276). */
int bhg_upload(bhg_context* ctx, const bh_particle64* particles, size_t n);
/* The same from device memory of the context's GPU. */
int bhg_upload_device(bhg_context* ctx, const void* particles, size_t n);
/* Several independent systems stored back to back: system s is
 * particles[offsets[s] .. offsets[s] + counts[s]).  Every count > 0. */
int bhg_upload_systems(bhg_context* ctx, const bh_particle64* particles, const uint64_t* counts, size_t nsys);
/* Copies the particles back (blocks until done).  After a walk the order is
 * Morton order per system, as step_particles returns it (integrate_ttg.h:107). */
int bhg_download(bhg_context* ctx, bh_particle64* out);
int bhg_download_device(bhg_context* ctx, void* out);
size_t bhg_num_particles(const bhg_context* ctx);

/* ---- systems joining and leaving (continuous batching) ---------------------
 *
 * The reference runs one simulation per process (main.cc:114-263); a server
 * keeps many resident in one context instead and advances them together
 * with bhg_step_systems.  Every system has a handle (bhg_upload* hands out
 * new ones in order, see bhg_system_ids).  A system's results never depend
 * on which others share the context: its tree, walk and sums only touch its
 * own particles. */

/* One Plummer sphere (scale radius a, total mass, centre, bulk velocity),
 * G = 1, truncated at 10a: the distribution of bhg_ic_plummer. */
typedef struct bhg_sphere {
  uint64_t n;
  double a;
  double mass;
  double centre[3];
  double bulk[3];
} bhg_sphere;

/* Grows the context's buffers now for up to `particles` particles in up to
 * `systems` systems, with the node slots they bring at max_leaf 16, so that
 * systems added later within those sizes neither allocate nor copy the
 * resident state.  Counts against the HBM budget (BHG_ENOMEM past it). */
int bhg_reserve(bhg_context* ctx, size_t particles, size_t systems);

/* Appends one system of n particles from host memory; its handle goes to
 * *id.  The resident systems keep their particles and parameters; the new
 * one starts with theta 0.5, eps2 0 and no kick/drift (bhg_set_system_params). */
int bhg_add_system(bhg_context* ctx, const bh_particle64* particles, size_t n, uint64_t* id);
/* Appends one system generated on the device: one sphere, or two (a merger)
 * stored one after the other, particle ids id0, id0 + 1, ...  The particles
 * come from a counter-based generator keyed by seed (the second sphere by
 * a key derived from it), so a request's initial conditions are its seed:
 * the same seed gives the same particles, bit for bit, on every call. */
int bhg_add_generated(bhg_context* ctx, const bhg_sphere* spheres, int nspheres, uint64_t seed, uint32_t id0,
                      uint64_t* id);
/* Removes k systems by handle; out (host, optional) receives their particles
 * back to back in the order of `handles` (blocks when given).  The others
 * keep their order, particles and parameters. */
int bhg_remove_systems(bhg_context* ctx, const uint64_t* handles, size_t k, bh_particle64* out);
size_t bhg_num_systems(const bhg_context* ctx);

/* ---- particle text on the device ----------------------------------------------
 *
 * read_csv (io.cc:122-178) and write_vtk (io.cc:180-195), done by the GPU:
 * the text crosses PCIe once and is parsed or written by kernels, bit for bit
 * as the reference reads and writes it. */

/* Parses CSV text (host memory, nbytes bytes; one particle per line:
 * id,mass,x,y,z,vx,vy,vz; blanks around fields, an optional '\r' at line
 * ends, blank lines skipped, an optional header line whose first field is not
 * an id, numbers converted exactly as std::from_chars does) and makes the
 * particles the context's only system, in file order.  A malformed line gives
 * BHG_EINVAL with the line number and text in bhg_last_error.  Replaces
 * read_csv + bhg_upload. */
int bhg_upload_csv(bhg_context* ctx, const char* text, size_t nbytes);
/* The same for text already in device memory of the context's GPU. */
int bhg_upload_csv_device(bhg_context* ctx, const void* text, size_t nbytes);
/* The same, appended as one more system (handle to *id). */
int bhg_add_csv(bhg_context* ctx, const char* text, size_t nbytes, uint64_t* id);
/* The system `handle` as write_vtk writes it (legacy VTK ASCII PolyData:
 * points, mass scalar, velocity vector; numbers as an ostream with default
 * settings writes them), in storage order.  *len receives the size in bytes;
 * out (host, cap bytes) receives the text unless it is NULL; a buffer smaller
 * than *len gives BHG_EINVAL.  Blocks until done. */
int bhg_snapshot_vtk(bhg_context* ctx, uint64_t handle, char* out, size_t cap, size_t* len);
/* The handles of the resident systems, in storage order (bhg_num_systems of them). */
int bhg_system_ids(const bhg_context* ctx, uint64_t* out);

/* ---- phases ---------------------------------------------------------------- */

/* build_flat_tree (flat_build_ttg.h:276-281) minus the multipoles: bounds and
 * domain (flat_build_ttg.h:93-113, domain.h:23-30), Morton keys
 * (flat_tree.h:104-125), (key, index) radix sort and gather
 * (flat_build_ttg.h:117-190), octree topology (flat_tree.h:144-289,
 * flat_build_ttg.h:194-273). */
int bhg_build_tree(bhg_context* ctx, unsigned max_leaf, uint32_t group_size);
/* finalize_node over all nodes (flat_tree.h:257-274, multipole.h:34-102). */
int bhg_compute_multipoles(bhg_context* ctx);
/* run_grouped_pass (grouped_ttg.h:297-323) with the integrate callback of
 * step_particles (integrate_ttg.h:74-77) fused: v += kick_dt*G*a, then, if
 * drift_dt != 0, x += drift_dt*v.  accel_out (host, optional): G*a of every
 * particle in the output (Morton) order, 3 doubles each (blocks).  missing
 * (optional) receives 0, the reference's "nodes opened without data" count,
 * which a single-GPU tree never has. */
int bhg_walk_forces(bhg_context* ctx, const bhg_force_params* fp, uint32_t target_size, double kick_dt,
                    double drift_dt, double* accel_out, uint64_t* missing);
/* kick_one/drift_one (integrate.h:15-16) with the accelerations of the last
 * walk: the unfused form of the integrate phase. */
int bhg_integrate(bhg_context* ctx, double kick_dt, double drift_dt);

/* One whole force evaluation of step_particles' grouped branch
 * (integrate_ttg.h:88-107): build + multipoles + walk with fused kick/drift.
 * Replayed from a captured CUDA graph once the sizes repeat. */
int bhg_step(bhg_context* ctx, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
             uint32_t target_size, double kick_dt, double drift_dt);
/* One evaluation of every system with the per-system theta, eps2, kick_dt
 * and drift_dt last given to bhg_set_system_params (fp supplies G, the
 * quadrupole switch and the precision; fp->eps2 is not used: a system with
 * eps2 0 gets the reference's r^2 = 0 self-term mask whatever the others
 * have). */
int bhg_step_systems(bhg_context* ctx, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
                     uint32_t target_size);
/* Asynchronous forms, for overlapping one context's copies with another's
 * evaluations (several contexts, each on its own stream, each holding some
 * of the systems: a system's result does not depend on the others in its
 * context).  bhg_step_systems_async enqueues the evaluation and returns;
 * bhg_download_async enqueues the copy (into pinned memory it does not block;
 * `out` must stay valid until bhg_sync).  bhg_sync waits for the context's
 * stream and reports the enqueued evaluations: BHG_OK; BHG_EAGAIN when the
 * octree outgrew its node slots (they are grown: the state is as after the
 * last evaluation that ran, and the message says how many ran); or the
 * error that stopped them.  A blocking step, or a call that changes the
 * systems, after async ones reports them first, as bhg_sync would. */
int bhg_step_systems_async(bhg_context* ctx, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
                           uint32_t target_size);
int bhg_download_async(bhg_context* ctx, bh_particle64* out);
int bhg_sync(bhg_context* ctx);
/* The leapfrog schedule of main.cc:199-246: a (dt/2, dt) evaluation,
 * steps-1 (dt, dt) evaluations and a closing (dt/2, 0) one. */
int bhg_run_schedule(bhg_context* ctx, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
                     uint32_t target_size, double dt, int steps);

/* Per-system parameters for a multi-system context (NULL arrays keep the
 * values given to bhg_step/bhg_walk_forces): theta, eps2, kick_dt, drift_dt. */
int bhg_set_system_params(bhg_context* ctx, const double* theta, const double* eps2, const double* kick_dt,
                          const double* drift_dt);

/* The particle cap of one walk group (1 .. 64; 0 = the default, 64).  The
 * walk runs one warp per group of consecutive walk targets of one system;
 * the group's targets share one traversal of the tree (each still gets
 * exactly the reference's own list, GroupWalker, grouped_ttg.h:204-289), so
 * larger groups share more, smaller ones give more groups to spread over
 * the GPU.  Results are reproducible bit for bit for a given cap. */
int bhg_set_walk_group(bhg_context* ctx, uint32_t particles);

/* Blocks.  reset != 0 starts new sums after reading. */
int bhg_get_stats(bhg_context* ctx, bhg_stats* out, int reset);
/* Device-side status bits of the last step (0 = fine); blocks. */
int bhg_device_status(bhg_context* ctx, uint32_t* status);

/* ---- inspection (parity tests) -------------------------------------------------- */

#define BHG_EXPORT_KEYS 1    /* uint64 sorted Morton keys [n] */
#define BHG_EXPORT_PERM 2    /* uint32 input index of each sorted particle [n] */
#define BHG_EXPORT_NODES_U32 3 /* uint32 [6][nodes]: begin, count, first_child, nchild, leaf, depth */
#define BHG_EXPORT_NODES_F64 4 /* double [nodes][14]: center xyz, hw, mass, com xyz, iab[6] */
#define BHG_EXPORT_DOMAINS 5 /* double [systems][4]: centre xyz, half width */
#define BHG_EXPORT_TARGETS 6 /* uint32 target node indices [targets] */
#define BHG_EXPORT_ACCEL 7   /* double [n][3]: G*a of the last walk, output order */
#define BHG_EXPORT_GROUPS 8  /* uint32 index (into the targets) of each walk group's first target [groups] */
/* Copies one of the arrays above to host memory (blocks).  bytes must be at
 * least the array's size; *written receives the size. */
int bhg_debug_export(bhg_context* ctx, int what, void* out, size_t bytes, size_t* written);

/* ---- diagnostics beside the path ------------------------------------------------ */

/* FP64 direct sum (brute_force.h:15-28) on the GPU for the sample rows
 * idx[0..ns) of the current (output-order) particles of system `sys`:
 * G*a into out[ns][3] (host).  Blocks. */
int bhg_direct_sum(bhg_context* ctx, int sys, const uint32_t* idx, size_t ns, double eps2, double G, double* out);
/* kinetic_energy / potential_energy (integrate.h:27-43; the potential is
 * unsoftened and O(N^2)) of system `sys` on the GPU.  Blocks. */
int bhg_energy(bhg_context* ctx, int sys, double G, double* kinetic, double* potential);

/* The energies of bhg_energy for callers that cannot allocate GPU memory
 * (a host program whose memory pool already owns the device, or a loop that
 * cannot afford the device-wide synchronisation of cudaFree).  No counterpart
 * in the reference.  particles: n records in device memory of the current
 * device; result: 2 doubles in device memory, written with (kinetic,
 * potential).  Allocates nothing: the per-block partial sums live in a fixed
 * 16 KB array in the library's device memory, so n is at most 262,144 (larger
 * n returns BHG_EINVAL).  Asynchronous on `stream` (a cudaStream_t; NULL =
 * the default stream).  The first call in a CUDA context (normally once per
 * device) looks up that array's device address: make it before any stream
 * capture; after cudaDeviceReset the next call looks it up again.  Errors:
 * BHG_ECUDA only for this call's own lookup or launches (an earlier,
 * unrelated error on the thread is neither reported nor cleared).  Every call shares the
 * array: calls that overlap on the GPU race and must be serialised (one
 * stream, or events between streams). */
int bhg_energy_noalloc(const bh_particle64* particles, size_t n, double G, double* result, void* stream);

/* Self-test of the give-up path of the bounded waits.  The radix sort and
 * the scans wait for their predecessor tiles' look-back words (decoupled
 * look-back); a wait that sees no word after a bounded number of polls stops,
 * sets a status bit and lets its kernel finish, so a stalled predecessor
 * gives BHG_EDEVICE instead of a hung GPU.  This runs that same wait on a
 * prepared array of 8 tile words, 1..7 published with an aggregate of 1 and
 * tile 0 published with an inclusive prefix of 1 (publish_first != 0) or never
 * published, with a poll limit of spin_limit (1 .. 2^20).  Never published:
 * the wait gives up and the call returns BHG_EDEVICE with the status text;
 * published: BHG_OK and *prefix (optional) = 8.  The context stays usable
 * either way.  No counterpart in the reference (its waits are TTG's). */
int bhg_selftest_wait(bhg_context* ctx, int publish_first, uint32_t spin_limit, uint32_t* prefix);

/* ---- workload generators (synthetic initial conditions) --------------------------- */

/* Plummer sphere by Aarseth-Henon-Wielen sampling (G = 1): n particles of
 * mass total_mass/n, scale radius a, radii below 10a, centred at centre[3]
 * with bulk velocity bulk[3].  Deterministic in `seed`; ids id0..id0+n-1.
 * Returns the next RNG state so a second sphere can continue the stream. */
uint64_t bhg_ic_plummer(bh_particle64* out, size_t n, double a, double total_mass, const double* centre,
                        const double* bulk, uint32_t id0, uint64_t seed);
/* Writes particles as the reference's CSV input (io.h:11-17). */
int bhg_write_csv(const char* path, const bh_particle64* p, size_t n);

/* Measured FP32 FMA throughput of the device (TFLOP/s, 2 flops per FMA):
 * a calibration loop of dependent-free FMAs on every SM. */
int bhg_measure_fp32_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* BHG_H */
