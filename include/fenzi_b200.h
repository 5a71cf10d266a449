/*
 * fenzi_b200 — C ABI of the B200-native FEN ZI molecular-dynamics step.
 *
 * The reference (TauferLab/fen-zi) has no plugin API: its boundary is a set of
 * `void f(void)` host functions on file-scope globals, called from main() in
 * src/fenzi.cu:141-268,442-547.  Each entry point below names the reference
 * function it replaces.  Differences in convention:
 *   - state lives behind an opaque fz_system* handle instead of globals;
 *   - every call returns an fz_status (the reference calls exit()); the detail
 *     of the last error on the calling thread is available from fz_last_error();
 *   - arrays are plain host pointers with explicit sizes; units are the
 *     reference's AKMA units (Angstrom, kcal/mol, amu, e, AKMA time for
 *     velocities: Angstrom per 1/20.4548 ps).
 * One handle must be used from one host thread at a time.
 */
#ifndef FENZI_B200_H
#define FENZI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int fz_status;
#define FZ_OK 0
#define FZ_ERR_IO 1        /* file missing / unreadable                     */
#define FZ_ERR_PARSE 2     /* malformed input, missing parameter            */
#define FZ_ERR_CUDA 3      /* CUDA runtime error                            */
#define FZ_ERR_CAPACITY 4  /* a device capacity was exceeded (list, cell)   */
#define FZ_ERR_SHAKE 5     /* SHAKE/RATTLE did not converge in its cap      */
#define FZ_ERR_ARG 6       /* bad argument                                  */
#define FZ_ERR_STATE 7     /* call out of order (e.g. step before upload)   */
#define FZ_ERR_NOMEM 8     /* device memory budget refused                  */
#define FZ_ERR_TIMEOUT 9   /* a bounded device wait ran out                 */

typedef struct fz_system fz_system;

/* Run-file settings, the keywords of ReadInput (src/prmread.cu:491-913). */
typedef struct fz_config {
  char coordinates[512];
  char structure[512];
  char parameters[512];
  char topology[512];
  char outputname[512];
  char outputtrajectory[512];
  char restartfilename[512];
  double temperature;        /* K */
  double thermostat;         /* "thermostat" (tau), stored, unused by NVE/reassignment */
  int temp_reset_every;      /* tempresetTiming: velocity reassignment period (0 = never) */
  int minimize_steps;
  double conjgradfac, steepdesfac, conjgradrate, steepdesrate;
  int start_step;
  double timestep_ps;        /* timestep (ps) */
  int dyna_steps;            /* dynasteps */
  double kappa;              /* KAPPa = Ewald beta (1/A) */
  int inbfrq;                /* INBFRQ: forced list rebuild period (0 = displacement-triggered) */
  int output_every;          /* outputTiming */
  int checkpoint_every;      /* checkpointTiming */
  int traj_every;            /* trajfrequencyTiming */
  double cuton, cutoff, pairlistdist;
  int gpublocksize;
  double box[3];             /* cellBasisVector1..3 diagonal */
  int pme_grid[3];           /* PMEGridSizeX/Y/Z */
  double pmass, pref;        /* Andersen piston mass, reference pressure (atm) */
  int shake;                 /* shake on|off */
  double shake_tol;
  double hfac;               /* hydrogen mass factor when shake is off */
  int printlevel, printtostdout, keepcheckpoints;
  char checkpointformat;     /* 'a' ascii, 'b' binary, 0 unset */
  long long seed;
  int unknown_keywords;      /* count of unrecognised lines (the reference warns) */
  /* restraints (src/prmread.cu:674-690): the mass centre of segment consharm_seg[1]
   * pulled towards that of consharm_seg[0] + consharm_dist with consharm_fc */
  int consharm;
  char consharm_seg[2][64];
  double consharm_dist[3];
  double consharm_fc;
  /* fixed segments (consfix, src/prmread.cu:697-723): their atoms never move */
  int consfix_nseg;
  char consfix_seg[8][64];
} fz_config;

/* Energies, the EvalProps table (src/evalprops.cu:248-308), kcal/mol, FP64. */
typedef struct fz_energies {
  double bond, angle, ureyb, dihed, impr, vdw, elec, pme, ewexcl, ewself;
  double potential;          /* sum of the above */
  double kinetic;            /* 1/2 sum m v^2 */
  double temperature;        /* 2 KE / (k_B (3N - 6 - Ncons)) */
  double virial[3];          /* diagonal of the virial sum r (x) F, constraint forces included (kcal/mol) */
  double pressure_atm;       /* (2 KE + W) / (3 V), src/cell_based_kernels.cu:582-587 */
  long long step;
  double box[3];             /* current box edges (A); they change under the barostat */
  double volume;             /* A^3 */
  double conserved;          /* KE + U, plus Pref V + piston kinetic energy under the barostat */
} fz_energies;

/* Sizes of a loaded system. */
typedef struct fz_info {
  int natom, ntypes, nbond, nangle, nureyb, ndihedral, nimproper;
  int nconstraint, ncluster, nexcl_pairs, n14_pairs;
  int ndihedral_terms;       /* dihedral rows after expanding multi-fold parameters */
  int pme_grid[3];
  double box[3];
} fz_info;

/* ---- errors ---------------------------------------------------------- */
/* Copies the last error message of this thread into buf (always NUL-terminated). */
fz_status fz_last_error(char* buf, size_t len);
const char* fz_version(void);

/* ---- input (host only, no GPU needed) ---------------------------------- */
/* ReadInput, src/prmread.cu:491-913.  Relative paths in the file stay relative
 * to the directory of in_path. */
fz_status fz_read_input(const char* in_path, fz_config* out);
/* LoadCoord (ReadCrd/ReadPdb/ReadXYZ, src/prmread.cu:285-488, picked by extension
 * as at src/prmread.cu:762-779), ReadPsf_CHARMM (:1442), ReadPrm_CHARMM (:2181),
 * build_constraints (:1303) and GenExcl_minimal_new (:2928), in that order. */
fz_status fz_load_system(const fz_config* cfg, fz_system** out);
fz_status fz_get_info(const fz_system* sys, fz_info* out);
/* Copies a named topology array (for inspection/tests): "pos" (double 3n), "q", "mass"
 * (double n), "type" (int n), "eps4","sig2","eps4_14","sig2_14" (double nt*nt),
 * "bond" (int 2nb), "bond_k","bond_r0", "angle" (int 3na), "angle_k","angle_t0",
 * "ureyb" (int 2), "ureyb_k","ureyb_r0", "dihe" (int 4nd, one row per fold),
 * "dihe_k","dihe_d" (double), "dihe_n" (int), "impr" (int 4ni), "impr_k","impr_p0",
 * "cons" (int 2nc), "cons_d", "excl" (int 2 x nexcl, 1-2/1-3 pairs), "p14" (int 2 x n14).
 * bytes must equal the array size. */
fz_status fz_get_array(const fz_system* sys, const char* name, void* out, size_t bytes);
fz_status fz_free(fz_system* sys);

/* ---- device ------------------------------------------------------------ */
/* InitMem (src/mem.cu:49) + InitDeviceConstants (src/cell_based_kernels.cu:1831):
 * allocates and fills device state on `device`; work is queued on `stream`
 * (a cudaStream_t, NULL = a stream owned by the system). */
fz_status fz_upload(fz_system* sys, int device, void* stream);
/* InitVelocity (src/init.cu:19-211): Maxwell-Boltzmann velocities at T (K) from a
 * counter-based generator keyed on (seed, counter), COM momentum removed, constraint
 * components removed (RATTLE). */
fz_status fz_reassign_velocities(fz_system* sys, double T, uint64_t seed, uint32_t counter);
/* ComputeAccelGPU (src/mdcuda.cu:557-849): forces at the current positions.  With
 * energies != 0 also evaluates the energy terms (read them with fz_eval_props). */
fz_status fz_compute_forces(fz_system* sys, int energies);
/* As fz_compute_forces, restricted to the selected terms (bitwise OR of FZ_TERM_*):
 * the real-space pair kernel (nonbondforce), the bonded kernel (bondedforce: bonds,
 * angles, Urey-Bradley, dihedrals, impropers, 1-4 pairs, Ewald exclusion correction)
 * and the PME reciprocal sum (ChargeSpread + FFT + BCMultiply + PMEForce). */
#define FZ_TERM_NONBONDED 1
#define FZ_TERM_BONDED 2
#define FZ_TERM_PME 4
#define FZ_TERM_ALL 7
/* Parts of FZ_TERM_BONDED, selectable one by one (the reference keeps one energy
 * array per part, src/bonded_forces.cu:597-640): bonds, angles, Urey-Bradley,
 * dihedrals, impropers, 1-4 pairs, Ewald exclusion correction.  Restraints come only
 * with FZ_TERM_BONDED. */
#define FZ_TERM_BONDS 8
#define FZ_TERM_ANGLES 16
#define FZ_TERM_UREYB 32
#define FZ_TERM_DIHEDRALS 64
#define FZ_TERM_IMPROPERS 128
#define FZ_TERM_PAIRS14 256
#define FZ_TERM_EXCLUSIONS 512
#define FZ_TERM_BONDED_PARTS 1016
fz_status fz_compute_forces_terms(fz_system* sys, int terms, int energies);
/* SingleStep (src/dynamics.cu:623-820) x nsteps: velocity Verlet with SHAKE/RATTLE,
 * device-side neighbour maintenance, velocity reassignment every temp_reset_every
 * steps when set.  Returns after the work is queued and checked. */
fz_status fz_step(fz_system* sys, int nsteps);
/* EvalProps (src/evalprops.cu:17-308): energies of the current state, with the
 * virial (force terms, PME reciprocal term and the instantaneous constraint forces)
 * and the pressure (src/evalprops.cu:214-218). */
fz_status fz_eval_props(fz_system* sys, fz_energies* out);
/* SaveCheckpointBinary/Ascii and LoadCheckpointBinary/Ascii (src/prmwrite.cu:31-252):
 * restart files in the reference's two layouts; format 'a' (ascii), 'b' (binary) or 0
 * (the input's checkpointformat, binary when unset).  Loading sets positions,
 * velocities, the step count, the seed and the box (and the barostat's box velocity);
 * the atom count must match. */
fz_status fz_checkpoint_save(fz_system* sys, const char* path, int format);
fz_status fz_checkpoint_load(fz_system* sys, const char* path, int format);
/* CHARMM DCD trajectory (charmm_trj_write_header/titles/natoms/frame,
 * src/io/charmmio.c; written every trjFreq steps by src/fenzi.cu:513-528): open writes
 * the header, write appends the system's current positions and unit cell, close
 * patches the frame count.  every = steps between frames (header only). */
typedef struct fz_dcd fz_dcd;
fz_status fz_dcd_open(fz_system* sys, const char* path, int every, fz_dcd** out);
fz_status fz_dcd_write(fz_dcd* traj);
fz_status fz_dcd_close(fz_dcd* traj);
/* MinimizeStep x minimizesteps (src/dynamics.cu:491-620, src/fenzi.cu:397-418):
 * conjugate-gradient moves (conjgradfac, conjgradrate) until the potential energy
 * rises, then steepest descent (steepdesfac, steepdesrate) until it rises again, at
 * most max_steps kept moves; a move that raised the energy is undone and not counted
 * (the first move is always kept, as in the reference); every 100 moves the current
 * factor is multiplied by its rate x 100; constraints are kept.  Velocities are
 * zeroed: call fz_reassign_velocities before dynamics.  Reports the moves kept and
 * the final potential energy (kcal/mol). */
fz_status fz_minimize(fz_system* sys, int max_steps, int* steps_done, double* energy_out);
/* Andersen constant-pressure dynamics for the following fz_step calls (the reference's
 * PCONSTANT build: src/cell_based_kernels.cu:566-579 piston acceleration,
 * src/mdcuda.cu:58-88 half kicks; keywords pref/pmass, src/prmread.cu:663-670).
 * The box keeps its aspect ratios; its x edge L follows
 * L'' = (P - pref) / (3 pmass L^2) - 2 L'^2 / L with P in kcal/mol/A^3.  Each
 * barostat step synchronises with the host once (the pressure steers the next box).
 * enable = 0 returns to constant volume at the current box. */
fz_status fz_set_barostat(fz_system* sys, int enable, double pref_atm, double pmass);
/* Host <-> device state (original atom order). */
fz_status fz_get_positions(fz_system* sys, double* out3n);
fz_status fz_set_positions(fz_system* sys, const double* in3n);
fz_status fz_get_velocities(fz_system* sys, double* out3n);
fz_status fz_set_velocities(fz_system* sys, const double* in3n);
/* Forces of the last evaluation (kcal/mol/A). */
fz_status fz_get_forces(fz_system* sys, double* out3n);
/* Bit-exact force accumulator (int64 fixed point, scale 2^32, x[n] y[n] z[n]). */
fz_status fz_get_forces_fixed(fz_system* sys, long long* out3n);
/* float32 state transfer through caller-pinned host buffers (x,y,z per atom). */
fz_status fz_set_state_f32(fz_system* sys, const float* pos3n, const float* vel3n);
fz_status fz_get_state_f32(fz_system* sys, float* pos3n, float* vel3n);
/* Device-side work counters: [0] kernel launches issued, [1] neighbour-list rebuilds,
 * [2] pair slots (i x j pairs the pair kernel evaluates per step, within or beyond the
 * cutoff) of the current pruned list, [3] list prunes. */
fz_status fz_get_counters(fz_system* sys, long long* out4);
/* Launch shapes in use: [0] pair tiles per pair-kernel work item (a fixed rule of the
 * tile count), [1] pair-kernel CTAs per SM, [2..4] PME brick edge per dimension
 * (charge-spread and gather block shape), [5] gather kernel (0 by atoms per brick, 1
 * one CTA per brick, 2 one thread per atom, 3 one thread per atom for the spread too,
 * without brick lists), [6] 1 when the autotuner picked [1..5]
 * at fz_upload (unless FZ_AUTOTUNE=0; every shape it can pick gives bit-identical
 * results).  No reference counterpart: the reference fixes its block sizes at
 * compile time (src/prmread.cu:109-115). */
fz_status fz_get_launch_shapes(fz_system* sys, int* out7);
/* Virial diagonal accumulated by the last fz_compute_forces_terms(..., energies = 1)
 * (force terms only: no constraint or kinetic part). */
fz_status fz_get_virial(fz_system* sys, double* out3);
/* Per-stage device timing (CUDA events on the system stream) for the steps run
 * while enabled.  Stages: 0 neighbour maintenance, 1 real-space pairs, 2 bonded,
 * 3 PME, 4 integrate (kick/drift/SHAKE + kick/RATTLE).  fz_get_stage_times returns
 * accumulated milliseconds per stage and the number of steps timed in out[5]. */
fz_status fz_set_stage_timing(fz_system* sys, int enable);
fz_status fz_get_stage_times(fz_system* sys, double* out6);
/* Measures this GPU's FP32 FMA throughput (TFLOP/s) with a register-resident FMA
 * kernel; the roof of the pair kernel, which no table of peaks carries. */
fz_status fz_measure_fp32_peak(int device, double* tflops);
/* No counterpart in the reference.  PME reciprocal-space forces (and optionally the
 * reciprocal energy) of n atoms for callers that cannot call cudaMalloc (code living
 * inside another framework's memory pool or a pre-sized arena).  Allocates nothing:
 * scratch lives in fixed file-scope device arrays (about 4.4 MB on each GPU that loads
 * the library, held until exit), and the per-call tables are computed on the device, so
 * nothing is copied from host memory.  pos4: device float4[n] (x, y, z, q); facc:
 * device int64[3n] fixed point (scale 2^32, x[n] y[n] z[n]), overwritten; energy_out:
 * host double or NULL (when given, the call synchronises `stream`).  Limits: n <=
 * 262144, grid sizes 2^a 3^b 5^c in 4..64.  The caller's current device is restored
 * on return.  The first call on a device resolves the scratch addresses (make it
 * before any stream capture); calls that overlap on the GPU race on the shared scratch
 * and must be serialised by the caller. */
fz_status fz_pme_reciprocal_static(int device, void* stream, const float* pos4, int n, const double* box,
                                   const int* K, double beta, long long* facc, double* energy_out);
/* ---- batched ensemble ------------------------------------------------- */
/* Independent uploaded systems (same device) advanced together: one MD step of every
 * system is one CUDA-graph launch whose branches are the systems' steps, so small
 * systems run concurrently on the GPU.  The batch does not own the systems; positions,
 * velocities and energies are read per system with the single-system calls. */
typedef struct fz_batch fz_batch;
fz_status fz_batch_create(fz_batch** out);
fz_status fz_batch_add(fz_batch* batch, fz_system* sys);
fz_status fz_batch_step(fz_batch* batch, int nsteps);
fz_status fz_batch_free(fz_batch* batch);
/* Removes a system (it keeps its device state and can be stepped alone or added again). */
fz_status fz_batch_remove(fz_batch* batch, fz_system* sys);
fz_status fz_batch_size(fz_batch* batch, int* out);

/* Serving loop (no counterpart in the reference, which runs one system per process):
 * a worker thread admits submitted jobs in FIFO order while the estimated device
 * memory of the running jobs stays within hbm_budget_bytes and fewer than max_running
 * run, keeps their state resident, advances the running mix together in the batch
 * graph in chunks of at most chunk_steps (a chunk ends when a job finishes), and
 * frees a job's device memory when it finishes, keeping its final energies and
 * positions.  Times are seconds since fz_server_create. */
typedef struct fz_server fz_server;
typedef struct fz_job_info {
  int job;
  int state;                 /* 0 queued, 1 running, 2 done, 3 failed */
  int status;                /* fz_status of a failed job */
  int natom;
  long long nsteps, steps_done;
  double submit_s, start_s, end_s;
  double device_bytes;       /* admission estimate */
  fz_energies final;         /* energies of the last frame (done jobs) */
} fz_job_info;
fz_status fz_server_create(int device, double hbm_budget_bytes, int chunk_steps, int max_running, fz_server** out);
/* Takes ownership of a loaded (not uploaded) system; it is freed by fz_server_free. */
fz_status fz_server_submit(fz_server* server, fz_system* sys, long long nsteps, int* job_id);
fz_status fz_server_info(fz_server* server, int job_id, fz_job_info* out);
/* Blocks until the job is done or failed; returns the job's status. */
fz_status fz_server_wait(fz_server* server, int job_id, fz_job_info* out);
/* Final positions (natom x 3, PSF order) of a done job. */
fz_status fz_server_positions(fz_server* server, int job_id, double* out);
/* [0] peak running jobs, [1] atom-steps done, [2] estimated bytes in use, [3] jobs finished. */
fz_status fz_server_stats(fz_server* server, double* out4);
/* The admission estimate of a loaded system's device memory (bytes). */
fz_status fz_server_estimate_bytes(const fz_system* sys, double* out);
/* Lets queued and running jobs finish, stops the worker, frees every job's system. */
fz_status fz_server_free(fz_server* server);
/* Synchronises the system's stream and reports any sticky device error status. */
fz_status fz_sync(fz_system* sys);
/* The system's CUDA stream (cudaStream_t), for callers that time or order work. */
void* fz_stream(fz_system* sys);

#ifdef __cplusplus
}
#endif
#endif
