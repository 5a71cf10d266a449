/* fenzi_plain: the "plain" single-system GPU path, a comparator for fenzi_b200.
 *
 * It restates the reference's own GPU algorithm stage for stage, one launch per
 * stage and a host synchronisation every step, so that fenzi_b200's step can be
 * timed against the reference's method on the same GPU:
 *   - cell list of edge >= pairlistdist and a per-atom FULL neighbour list (each
 *     pair kept by both atoms, no Newton's third law), rebuilt when an atom has moved
 *     more than half the skin; the displacement test is read on the host every step
 *     (BuildNBGPU, src/dynamics.cu:237-341; the rebuild decision, src/dynamics.cu:695-737);
 *   - thread-per-atom nonbonded force over that list (nonbondforce,
 *     src/nonbonded_forces.cu:25-270);
 *   - thread-per-term bonded forces with atomics (bondedforce, src/bonded_forces.cu:597-1381);
 *   - PME with per-grid-point atom lists built by atomics and a gather-style spread
 *     (LatticeBuild/LatticeUpdate + ChargeSpread, src/cell_based_kernels.cu:1557-1767,
 *     src/pme_kernels.cu:20-239), two complex-to-complex cuFFT transforms
 *     (src/mdcuda.cu:748,780), the influence-function multiply (BCMultiply,
 *     src/cell_based_kernels.cu:1770-1826) and a thread-per-atom gather
 *     (PMEForce, src/pme_kernels.cu:381-770);
 *   - velocity Verlet with per-cluster SHAKE/RATTLE (SingleStep, src/dynamics.cu:623-820).
 * Forms and units are fenzi_b200's (CHARMM switch, erfc real-space Ewald, analytic
 * order-4 B-splines), so both paths agree with the same FP64 oracle.
 *
 * Arithmetic is FP32 (fp64 = 0; the reference's precision) or FP64 throughout
 * (fp64 = 1; the all-FP64 GPU variant used for energy-drift comparisons).
 * Not covered: barostat, restraints, fixed atoms, minimiser, velocity reassignment
 * (the caller sets velocities).  Arrays are in PSF atom order, AKMA units.
 *
 * Link: fenzi_b200/libfenzi_plain.so (needs libfenzi_b200.so and cuFFT). */
#ifndef FENZI_PLAIN_H
#define FENZI_PLAIN_H

#include "fenzi_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fz_plain fz_plain;

/* Device copy of a loaded system (fz_load_system; it need not be uploaded).
 * Positions start at the system's coordinates, velocities at zero. */
fz_status fz_plain_create(const fz_system* sys, int device, int fp64, fz_plain** out);
fz_status fz_plain_free(fz_plain* p);

fz_status fz_plain_set_positions(fz_plain* p, const double* in3n);
fz_status fz_plain_set_velocities(fz_plain* p, const double* in3n);
fz_status fz_plain_get_positions(fz_plain* p, double* out3n);
fz_status fz_plain_get_velocities(fz_plain* p, double* out3n);

/* ComputeAccelGPU: all forces at the current positions (rebuilding the lists
 * first when due); out3n may be NULL. */
fz_status fz_plain_compute_forces(fz_plain* p, double* out3n);

/* SingleStep x nsteps (one host synchronisation per step, as the reference). */
fz_status fz_plain_step(fz_plain* p, int nsteps);

/* EvalProps: energies of the current state (virial, pressure and box fields are
 * left at zero / the fixed box). */
fz_status fz_plain_eval_props(fz_plain* p, fz_energies* out);

/* out4: neighbour-list rebuilds, list entries (sum over atoms) at the last build,
 * steps taken, kernel launches issued. */
fz_status fz_plain_get_counters(fz_plain* p, long long* out4);

#ifdef __cplusplus
}
#endif
#endif
