/*
 * hpdmk.h — drop-in C interface of the B200 periodic DMK energy library.
 *
 * Mirrors the reference's include/hpdmk.h (PDMK4MC): the same enum
 * hpdmk_init (include/hpdmk.h:6-9), struct HPDMKParams with the same fields,
 * defaults and layout (include/hpdmk.h:11-17), the opaque handle hpdmk_tree
 * (include/hpdmk.h:19) and hpdmk_tree_create with the same signature
 * (include/hpdmk.h:25). The handle-based calls below expose what the
 * reference's C++ class HPDMKPtTree<double> offers (include/tree.hpp:74-132):
 * construction from positions and charges, form_outgoing_pw,
 * form_incoming_pw, eval_energy, eval_shift_energy and update_shift.
 *
 * Units and conventions follow the reference: positions are xyz-interleaved
 * in [0, L)^3, particle indices are the caller's original indices, energies
 * are E = 1/2 sum' q_i q_j / r over periodic images (no 4 pi).
 *
 * Every call returns an int status (HPDMK_OK = 0) where the reference threw.
 */
#ifndef HPDMK_H
#define HPDMK_H

#include <stddef.h>

#if defined(HPDMK_WITH_MPI)
#include <mpi.h>
#else
/* The library runs on one rank; without MPI the communicator is an opaque int. */
typedef int MPI_Comm;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD 0
#endif
#endif

#ifdef __cplusplus
typedef enum : int {
  DIRECT = 1,
  PROXY = 2,
} hpdmk_init;

typedef struct HPDMKParams {
  int n_per_leaf = 200;       /* maximum number of particles per leaf */
  int digits = 3;             /* 3, 6, 9 or 12 digits of accuracy */
  double L;                   /* side of the periodic cube */
  double prolate_order = 16;  /* kept for layout compatibility; unused */
  hpdmk_init init = PROXY;    /* DIRECT or PROXY (PROXY is limited to 3 digits, as in the reference) */
} HPDMKParams;
#else
typedef enum {
  DIRECT = 1,
  PROXY = 2,
} hpdmk_init;

typedef struct HPDMKParams {
  int n_per_leaf;
  int digits;
  double L;
  double prolate_order;
  hpdmk_init init;
} HPDMKParams;
#endif

typedef void *hpdmk_tree;

/* status codes */
#define HPDMK_OK 0
#define HPDMK_ERR_BAD_PARAMS 1     /* digits not in {3,6,9,12}, L <= 0, n_per_leaf < 1, PROXY with digits > 3 */
#define HPDMK_ERR_BAD_INPUT 2      /* n < 1, null pointer, position outside [0,L), non-finite value, index out of range */
#define HPDMK_ERR_CUDA 4           /* CUDA runtime failure (message via hpdmk_last_error_message) */
#define HPDMK_ERR_OUT_OF_MEMORY 5  /* device allocation failed */
#define HPDMK_ERR_DEVICE 6         /* device-side error word set (overflow pool exhausted, a bounded wait in a kernel gave up) */
#define HPDMK_ERR_INTERNAL 7

/* precision modes of hpdmk_tree_init_ext.
 * HPDMK_PRECISION_FP64: every step in FP64 (the drop-in path).
 * HPDMK_PRECISION_MIXED: the outgoing plane-wave expansions (root and boxes,
 * the reference's outgoing_pw_root / outgoing_pw_direct, src/planewave.cpp:24-84)
 * are formed on the tensor cores (tcgen05, kind::i8) from 8-bit slices: each
 * operand is a 32-bit fixed point written as four signed base-256 digits, the
 * ten slice products of order <= 3 are summed exactly in 32-bit integers and
 * combined in FP64, a coefficient error near 1e-9 of the box's largest
 * coefficient (energies within about 1e-9 of the FP64 path); the incoming
 * expansions, energy sums, near field, energy shifts and updates stay FP64. */
#define HPDMK_PRECISION_FP64 0
#define HPDMK_PRECISION_MIXED 1

typedef struct HPDMKExtParams {
  int leaf_slack;     /* free particle slots per leaf kept for moves (default 8) */
  int pool_capacity;  /* overflow slots for arrivals into full leaves (default 4096) */
  int precision;      /* HPDMK_PRECISION_FP64 (default) or HPDMK_PRECISION_MIXED */
  int device;         /* CUDA device ordinal (default 0) */
  void *stream;       /* cudaStream_t to run on; NULL: the tree creates its own */
} HPDMKExtParams;

#ifdef __cplusplus
extern "C" {
#endif

/* Reference: include/hpdmk.h:25, src/hpdmk.cpp:18-20 — builds the tree and
 * discards it (the reference's only C entry point). */
void hpdmk_tree_create(MPI_Comm comm, HPDMKParams params, int n_src, const double *r_src, const double *charge);

/* Reference: HPDMKPtTree(comm, params, r_src, charge), include/tree.hpp:74 and
 * src/tree.cpp:267-444. Copies r_src[3n] and charge[n] to the device.
 * Returns NULL on failure; hpdmk_last_error() tells why. */
hpdmk_tree hpdmk_tree_init(MPI_Comm comm, HPDMKParams params, int n_src, const double *r_src, const double *charge);

/* As hpdmk_tree_init, with library extensions; ext may be NULL. */
hpdmk_tree hpdmk_tree_init_ext(MPI_Comm comm, HPDMKParams params, const HPDMKExtParams *ext, int n_src,
                               const double *r_src, const double *charge);

/* As hpdmk_tree_init_ext with d_r_src[3n] and d_charge[n] already in device memory.
 * Positions and charges are validated on the device during the build; a
 * position outside [0, L) or a non-finite charge returns NULL with
 * HPDMK_ERR_BAD_INPUT. The arrays are read on the tree's stream and are no
 * longer needed once the call returns. */
hpdmk_tree hpdmk_tree_init_device(MPI_Comm comm, HPDMKParams params, const HPDMKExtParams *ext, int n_src,
                                  const double *d_r_src, const double *d_charge);

void hpdmk_tree_destroy(hpdmk_tree tree);

/* Reference: form_outgoing_pw (include/tree.hpp:102, src/planewave.cpp:86-97). */
int hpdmk_form_outgoing_pw(hpdmk_tree tree);

/* Reference: form_incoming_pw (include/tree.hpp:103, src/planewave.cpp:99-155). */
int hpdmk_form_incoming_pw(hpdmk_tree tree);

/* Reference: eval_energy = eval_energy_window + eval_energy_diff + eval_energy_res
 * (include/tree.hpp:105-108, src/energy.cpp:21-173). Any of the part pointers may be NULL. */
int hpdmk_eval_energy(hpdmk_tree tree, double *energy, double *window, double *difference, double *residual);

/* Convenience: form_outgoing_pw + form_incoming_pw + eval_energy. */
int hpdmk_energy(hpdmk_tree tree, double *energy);

/* Reference: eval_shift_energy(i, dx, dy, dz) (include/tree.hpp:122, src/energy_shift.cpp:18-70):
 * energy change of moving original particle i by (dx,dy,dz), wrapped into the box. */
int hpdmk_eval_shift_energy(hpdmk_tree tree, long i, double dx, double dy, double dz, double *dE);

/* Reference: update_shift(i, dx, dy, dz) (include/tree.hpp:132, src/tree.cpp:447-597):
 * commit the move; meant to follow hpdmk_eval_shift_energy with the same arguments
 * (the move is re-evaluated when the arguments differ). */
int hpdmk_update_shift(hpdmk_tree tree, long i, double dx, double dy, double dz);

/* Batched extension: dE[c] for m candidate moves (i[c], d[3c..3c+2]) against the
 * current state; no state change. Host arrays. */
int hpdmk_eval_shift_energy_batch(hpdmk_tree tree, int m, const long *i, const double *d, double *dE);

/* As hpdmk_eval_shift_energy_batch with device-resident int32 indices d_i[m],
 * displacements d_d[3m] and output d_dE[m], enqueued on the tree's stream
 * without a host synchronisation (one launch, one thread block per candidate). */
int hpdmk_eval_shift_energy_batch_device(hpdmk_tree tree, int m, const int *d_i, const double *d_d, double *d_dE);

/* No reference counterpart. The same single launch as
 * hpdmk_eval_shift_energy_batch (one thread block per candidate, phase tables
 * in shared memory), so the same results bit for bit, but the call allocates
 * no device memory: the candidates' indices and displacements and their
 * energy shifts are staged through one fixed static device array (144 KB per
 * device, its address looked up once per device). For callers that may not
 * allocate device memory once the tree exists: a process that budgets its
 * device memory up front, or one whose memory is handed out by another
 * framework's pool that it must not grow or bypass.
 * Limits: m <= HPDMK_STATIC_MAX_MOVES; larger m returns HPDMK_ERR_BAD_INPUT
 * with a message and does no work. Nothing in the array has to start at zero
 * (each call writes the inputs it reads). Calls that overlap in time on one
 * device share the array and race: make them one after another. Make the
 * first call on each device before any stream capture starts, since it looks
 * up the array's address. */
#define HPDMK_STATIC_MAX_MOVES 4096
int hpdmk_eval_shift_energy_batch_static(hpdmk_tree tree, int m, const long *i, const double *d, double *dE);

/* Batched extension: n sequential Metropolis moves at inverse temperature beta.
 * Move c proposes (i[c], d[3c..]) and is accepted when u[c] < exp(-beta dE);
 * accepted moves are committed before the next one. Outputs dE[c], accepted[c]
 * (either may be NULL). Host arrays. */
int hpdmk_mc_run(hpdmk_tree tree, int n, const long *i, const double *d, const double *u, double beta, double *dE,
                 int *accepted);

/* Replica sets (no reference counterpart): the Metropolis sequences of
 * n_trees independent trees (same digits setting, same device) in one
 * launch, one thread block per tree. Tree t runs moves c = 0 .. m-1 taken
 * from i[t m + c], d[3 (t m + c) ..], u[t m + c]; outputs dE and accepted
 * (either may be NULL) in the same layout. Same results as hpdmk_mc_run on
 * each tree, to rounding. Host arrays. */
int hpdmk_replicas_mc_run(int n_trees, const hpdmk_tree *trees, int m, const long *i, const double *d,
                          const double *u, double beta, double *dE, int *accepted);

/* Replica sets: form_outgoing_pw + form_incoming_pw + eval_energy of each
 * tree, energy[t], with several trees in flight at once (each on its own
 * stream, driven by a pool of host threads). No reference counterpart. */
int hpdmk_replicas_energy(int n_trees, const hpdmk_tree *trees, double *energy);

/* How hpdmk_mc_run / hpdmk_mc_run_device execute the sequence (no reference
 * counterpart): HPDMK_MC_PERSISTENT (default) runs it as one cooperative
 * launch on every SM with grid barriers between the phases of a move;
 * HPDMK_MC_GRAPH runs CUDA graphs of 128 (shift, update) launch pairs.
 * Both give the same results to rounding. */
#define HPDMK_MC_PERSISTENT 0
#define HPDMK_MC_GRAPH 1
int hpdmk_set_mc_mode(hpdmk_tree tree, int mode);

/* As hpdmk_mc_run with device-resident int32 indices and device outputs, enqueued on
 * the tree's stream without a host synchronisation (stream may be NULL for the default). */
int hpdmk_mc_run_device(hpdmk_tree tree, int n, const int *d_i, const double *d_d, const double *d_u, double beta,
                        double *d_dE, int *d_accepted);

/* Potentials and fields (no counterpart in the reference, which evaluates
 * energies only): phi[c] = dE/dq at particle i[c], the potential of all other
 * particles and of the periodic images of all particles including its own,
 * so that E = 1/2 sum_i q_i phi_i; field[3c..3c+2] = -grad phi there (may be
 * NULL; the force on the particle is its charge times the field). The same
 * expansions and near field as an energy shift; one launch for all m. */
int hpdmk_eval_potential(hpdmk_tree tree, int m, const long *i, double *phi, double *field);

/* Tree maintenance (no counterpart in the reference, which keeps the tree
 * built at construction and patches only its two lowest levels on moves,
 * src/tree.cpp:583-596): rebuild the octree, its neighbour lists and the
 * outgoing and incoming expansions from the current particle positions, so
 * that leaves are back at n_per_leaf after many moves. The handle and the
 * particles' original indices stay; the result equals a tree built from
 * hpdmk_get_positions. Runs on the device. */
int hpdmk_tree_rebuild(hpdmk_tree tree);

/* Rebuild policy: with leaf_factor > 1, every hpdmk_form_outgoing_pw first
 * checks how far the tree has drifted from the refinement rule under the
 * accepted moves and rebuilds it (as hpdmk_tree_rebuild, before forming the
 * outgoing expansions) when a leaf holds more than leaf_factor * n_per_leaf
 * particles or a refined node below level 2 holds fewer than
 * n_per_leaf / leaf_factor. Both thresholds are widened to the tree's own
 * values when the policy was set or the tree last rebuilt (leaves at the
 * level cap may hold more than n_per_leaf, nodes refined for the 2:1 balance
 * fewer), so a tree as built never triggers it. leaf_factor = 0 (the
 * default) turns the check off. The check is one small kernel and one
 * read-back per full energy. */
int hpdmk_set_rebuild_policy(hpdmk_tree tree, double leaf_factor);

/* The drift the policy looks at: the largest particle count of a leaf and
 * the smallest of a refined node below level 2 (n if there is none), from
 * the counts the moves maintain; *rebuilds = rebuilds the policy made. */
int hpdmk_tree_drift(hpdmk_tree tree, int *max_leaf, int *min_refined, int *rebuilds);

/* FP64 Ewald energy of the current particles, the comparator for the DMK
 * energy (reference: the Ewald summation of src/ewald.cpp:17-223, there on
 * the CPU): real-space erfc sum with the cut-off at one tree level's box size,
 * reciprocal sum over the structure factor, self term; truncation near 1e-12
 * relative. parts (may be NULL) receives real, reciprocal and self terms. */
int hpdmk_ewald_energy(hpdmk_tree tree, double *energy, double *parts);

/* Current positions in the caller's original order, r[3n]. */
int hpdmk_get_positions(hpdmk_tree tree, double *r);

/* Tree shape: info[0] number of levels, info[1] nodes, info[2] particles,
 * info[3] window modes, info[4] difference modes per box. */
int hpdmk_tree_info(hpdmk_tree tree, long *info);

/* Wait for all queued work of the tree. */
int hpdmk_synchronize(hpdmk_tree tree);

/* The CUDA stream (cudaStream_t) all work of the tree is enqueued on. */
int hpdmk_get_stream(hpdmk_tree tree, void **stream);

/* Kernel timing: with enable != 0, CUDA events bracket every shift, update,
 * persistent Metropolis and outgoing-expansion launch on the tree's stream
 * (graph-run updates: a 1-in-8 sample of the batches). hpdmk_get_timing
 * synchronises and returns, per kernel class c (0 shift, 1 update, 2 persistent
 * Metropolis launch, 3 outgoing NUDFT), out[2c] = total milliseconds and
 * out[2c+1] = number of launches since the last reset. */
int hpdmk_set_timing(hpdmk_tree tree, int enable);
int hpdmk_get_timing(hpdmk_tree tree, double *out, int reset);

/* Work counters of the last MC batch: out[0] accepted moves, out[1] bytes of
 * expansion data read+written by their updates (algorithmic: 32 B per complex RMW),
 * out[2] algorithmic bytes read by the dE evaluations of the persistent kernel. */
int hpdmk_get_update_bytes(hpdmk_tree tree, double *out);

/* Autotuner (no reference counterpart): times the energy pipeline of this
 * tree over candidate run-time splits and tiles, one parameter at a time,
 * with CUDA events on the tree's stream, keeps the fastest and records them
 * per (digits, precision, floor(log2 N)) in the JSON table at `path` (NULL
 * or "": tuning.json beside the library, or the file named by the
 * environment variable HPDMK_TUNING). New trees read that table. The
 * parameters, chosen[0..3]: particles per split-K chunk of a box in the
 * outgoing pass, particles per chunk of the root pass, resident waves of
 * blocks in the incoming pass, most near-field target chunks per leaf;
 * times[0..2] (may be NULL): outgoing, incoming and near-field milliseconds
 * with the chosen values (medians of `reps` runs). The tree's expansions are
 * left formed. */
int hpdmk_autotune(hpdmk_tree tree, const char *path, int reps, int *chosen, double *times);
/* The tree's current run-time splits and tiles (the four values above), and
 * setting them by hand (values are clamped to the supported ranges). */
int hpdmk_get_tuning(hpdmk_tree tree, int *out);
int hpdmk_set_tuning(hpdmk_tree tree, const int *in);

/* Kernel launches this library has issued since it was loaded, kernels run
 * inside its captured CUDA graphs included (no reference counterpart). */
int hpdmk_get_launch_count(long long *out);

/* Reference: read_particle_info (src/utils.cpp:14-28). Reads a text file
 * whose first line is a header and whose further lines hold "x y z q"
 * (whitespace-separated; lines that do not start with four numbers are
 * skipped). *n receives the number of particles. With r and q both NULL the
 * call only counts; otherwise r[3 n] (xyz-interleaved) and q[n] are filled,
 * and capacity (particles) must be at least *n. Host only, no device work. */
int hpdmk_read_particle_info(const char *filename, long *n, double *r, double *q, long capacity);

/* Last status of the calling thread and its message. */
int hpdmk_last_error(void);
const char *hpdmk_last_error_message(void);

/* Introspection used by the parity tests (not part of the reference interface). */
int hpdmk_debug_nodes(hpdmk_tree tree, int *level, unsigned long long *prefix, int *is_leaf, long *count);
int hpdmk_debug_neighbors(hpdmk_tree tree, int *colleague27, int *coarse8);
int hpdmk_debug_sorted_order(hpdmk_tree tree, long *orig_of_sorted);
int hpdmk_debug_pw(hpdmk_tree tree, long node, int which, double *out);
int hpdmk_debug_kernels(hpdmk_tree tree, int level, double *out);
int hpdmk_debug_shift_parts(hpdmk_tree tree, long i, double dx, double dy, double dz, double *parts);
/* Host-only PSWF set-up for a digits setting: out[0] c, out[1] lambda, out[2] C0 / psi0(0),
 * out[3] diff0, out[4] n_window, out[5] n_diff; psi[k] = psi0(x[k]) / psi0(0) for k < nx. */
int hpdmk_debug_prolate(int digits, double *out, int nx, const double *x, double *psi);
/* Host-only: the tuning a tree of (digits, precision, n) would read from the table file at path. */
int hpdmk_debug_tuning_lookup(const char *path, int digits, int precision, long n, int *out);

#ifdef __cplusplus
}
#endif

#endif /* HPDMK_H */
