/*
 * ffxcuda.h -- C ABI of the B200 AMOEBA energy/gradient library (libffxcuda.so).
 *
 * This is the drop-in boundary for Force Field X's AMOEBA polarizable
 * energy-and-gradient path.  A Java `CudaForceFieldEnergy extends
 * ForceFieldEnergy` (selected through the `platform` key in
 * ForceFieldEnergy.energyFactory, modules/potential/.../ForceFieldEnergy.java:1464-1510,
 * the same plug point OpenMMEnergy uses, modules/potential/.../openmm/OpenMMEnergy.java:80)
 * binds these symbols with the JDK Foreign Function & Memory API.
 *
 * Conventions
 *  - Plain C types only; every array is a caller-owned host buffer.  The
 *    library copies in and out and never retains a caller pointer.
 *  - Units follow Force Field X: Angstrom, electron, kcal/mol.  Multipoles are
 *    passed in e, e*A, e*A^2 (already converted from the Bohr units of the
 *    parameter file, MultipoleType.java:1115-1119), in the order
 *    t000,t100,t010,t001,t200,t020,t002,t110,t101,t011 (MultipoleType.java:109-137).
 *  - Every call returns an ffxg_status; 0 is success.  Java maps a nonzero
 *    status to EnergyException (ffx/potential/utils/EnergyException.java), as the
 *    reference throws at PCGSolver.java:554-568 and RealSpaceEnergyRegion.java:384-391.
 *  - One handle owns one CUDA stream.  Calls on one handle must be serialised
 *    by the caller; distinct handles may be used concurrently.
 *  - There is no CPU fallback: if no sm_100 device is present, ffxg_create
 *    returns FFXG_ERR_CUDA.
 */
#ifndef FFXCUDA_H
#define FFXCUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ffxg_handle ffxg_handle;

typedef enum {
  FFXG_OK = 0,
  FFXG_ERR_BAD_ARG = 1,       /* invalid argument / unsupported configuration */
  FFXG_ERR_CUDA = 2,          /* CUDA runtime error or no usable device */
  FFXG_ERR_SCF_DIVERGED = 3,  /* PCG residual grew (PCGSolver.java:547-559) */
  FFXG_ERR_SCF_MAXITER = 4,   /* PCG hit the iteration cap (PCGSolver.java:563-568) */
  FFXG_ERR_NONFINITE = 5,     /* NaN/Inf energy, torque or gradient */
  FFXG_ERR_CAPACITY = 6,      /* neighbour capacity exceeded even after regrowth */
  FFXG_ERR_RANGE = 7          /* mixed form only: a fixed-point (2^-32) force, torque or mesh
                                 sum reached 2^20 in magnitude.  Every output is written and
                                 accurate to FP64 rounding, but no longer guaranteed to repeat
                                 bit for bit; callers may treat it as a warning. */
} ffxg_status;

/* Local multipole frame definitions (MultipoleType.MultipoleFrameDefinition). */
typedef enum {
  FFXG_FRAME_NONE = 0,
  FFXG_FRAME_ZONLY = 1,
  FFXG_FRAME_ZTHENX = 2,
  FFXG_FRAME_BISECTOR = 3,
  FFXG_FRAME_ZTHENBISECTOR = 4,
  FFXG_FRAME_THREEFOLD = 5
} ffxg_frame;

typedef enum {
  FFXG_PRECISION_FP64 = 0,    /* plain FP64 form: the reference's arithmetic */
  FFXG_PRECISION_MIXED = 1    /* FP32 pair tensors/splines/FFT, FP64 PCG scalars and energies */
} ffxg_precision;

typedef enum {
  FFXG_POLAR_NONE = 0,
  FFXG_POLAR_DIRECT = 1,
  FFXG_POLAR_MUTUAL = 2
} ffxg_polarization;

/* Energy terms returned by ffxg_energy (kcal/mol). */
enum {
  FFXG_TERM_VDW = 0,
  FFXG_TERM_PERMANENT = 1,       /* real + self + reciprocal + charge correction */
  FFXG_TERM_POLARIZATION = 2,    /* real + self + reciprocal */
  FFXG_TERM_PERM_REAL = 3,
  FFXG_TERM_PERM_SELF = 4,
  FFXG_TERM_PERM_RECIP = 5,
  FFXG_TERM_POL_REAL = 6,
  FFXG_TERM_POL_SELF = 7,
  FFXG_TERM_POL_RECIP = 8,
  FFXG_TERM_TOTAL = 9,
  FFXG_N_TERMS = 10
};

/* Interaction counts returned by ffxg_energy. */
enum {
  FFXG_COUNT_VDW = 0,          /* VanDerWaals.getInteractions (VanDerWaals.java:583) */
  FFXG_COUNT_PERMANENT = 1,    /* ParticleMeshEwald.getInteractions (ParticleMeshEwald.java:1014) */
  FFXG_COUNT_SCF_ITER = 2,     /* completed PCG cycles (PCGSolver.scfByPCG return value) */
  FFXG_COUNT_LIST_BUILDS = 3,  /* neighbour-list rebuilds performed during this call */
  FFXG_COUNT_LIST_PAIRS = 4,   /* unordered pairs in the buffered neighbour list (the CPU
                                  oracle fills it; the library writes -1 and returns the pair
                                  set through ffxg_get_neighbor_pairs) */
  FFXG_COUNT_LIST_GROWTHS = 5, /* list capacity regrowths during this call: a row overflowed
                                  its capacity, the rows grew by half and the evaluation was
                                  repeated (the result is that of the repeat) */
  FFXG_N_COUNTS = 6
};

/* Resolved per-atom topology and parameters.  This is exactly the data that
 * ParticleMeshEwald and VanDerWaals hold after assignment: localMultipole,
 * frame/axisAtom (ParticleMeshEwald.java:2535-2600), polarizability / thole /
 * ipdamp (:1395-1410), mask12..mask15 and ip11 (:1414-1445, :2616-2650), and the
 * vdW class tables (VanDerWaalsForm.java:355-470). */
typedef struct {
  int32_t n_atoms;
  const double *xyz;             /* [n][3] coordinates */
  const double *multipole;       /* [n][10] local-frame multipoles */
  const int32_t *frame;          /* [n] ffxg_frame */
  const int32_t *axis;           /* [n][3] frame-defining atoms (z, x, y), -1 = unused */
  const double *polarizability;  /* [n] A^3 */
  const double *thole;           /* [n] Thole damping parameter */
  const double *pdamp;           /* [n] polarizability^(1/6); <= 0 disables damping */
  const int32_t *vdw_type;       /* [n] row of the vdW pair tables */
  const int32_t *red_parent;     /* [n] heavy atom for hydrogen reduction (self if none) */
  const double *red_factor;      /* [n] reduction factor (0 if none) */
  int32_t n_vdw_types;
  const double *vdw_inv_rmin;    /* [t][t] 1 / combined Rmin (0 = no interaction) */
  const double *vdw_eps;         /* [t][t] combined well depth */
  /* Bonded relationship lists in CSR form: ptr[n+1], idx[ptr[n]]. */
  const int32_t *mask12_ptr, *mask12_idx;
  const int32_t *mask13_ptr, *mask13_idx;
  const int32_t *mask14_ptr, *mask14_idx;
  const int32_t *mask15_ptr, *mask15_idx;
  const int32_t *ip11_ptr, *ip11_idx;   /* polarization group of each atom (includes itself) */
} ffxg_system;

typedef struct {
  double box[3];                 /* cell edges a, b, c (A); angles below */
  double vdw_cutoff;             /* A (vdw-cutoff) */
  double vdw_taper;              /* fraction of the cutoff where the taper starts (vdw-taper, 0.9) */
  double ewald_cutoff;           /* A (ewald-cutoff) */
  double ewald_alpha;            /* 1/A (ewald-alpha) */
  double list_buffer;            /* A (list-buffer, 2.0) */
  int32_t pme_grid[3];           /* PME mesh dimensions, 5 .. 4096 each (any factors: radices 2-7 have
                                    their own butterflies, larger primes a general pass) */
  int32_t pme_order;             /* B-spline order (5) */
  double polar_eps;              /* PCG convergence, Debye RMS (polar-eps) */
  int32_t max_scf_iter;          /* PCG iteration cap (1000 in the reference) */
  int32_t polarization;          /* ffxg_polarization */
  double precond_cutoff;         /* cg-preconditioner-cutoff (4.5) */
  double precond_scale;          /* cg-preconditioner-scale (2.0) */
  double electric;               /* 332.0637133 */
  double m12, m13, m14, m15;     /* mpole-1n-scale */
  double p12, p13, p14, p15;     /* polar-1n-scale */
  double intra14;                /* polar-14-intra */
  double d11;                    /* direct-11-scale */
  double v12, v13, v14;          /* vdw-1n-scale */
  int32_t precision;             /* ffxg_precision */
  double angles[3];              /* cell angles alpha, beta, gamma (degrees; 0 reads as 90).  With box
                                    (a, b, c) they give the cell of Crystal.updateCrystal
                                    (C/Crystal.java:1428-1548): orthorhombic, monoclinic (only beta
                                    differs from 90) or general.  The pair lists need every
                                    interaction cutoff below half of each perpendicular width, or
                                    take lists of every lattice image. */
} ffxg_params;

/* Build a handle: validate the system, upload topology and parameters, pick a
 * device, allocate device buffers.  Replaces the ForceFieldEnergy /
 * ParticleMeshEwald / VanDerWaals constructors (ForceFieldEnergy.java:1207-1245,
 * ParticleMeshEwald.java:490-741, VanDerWaals.java:308-404). */
int ffxg_create(const ffxg_system *sys, const ffxg_params *params, ffxg_handle **out);

/* Release every device resource held by the handle. */
void ffxg_destroy(ffxg_handle *h);

/* Last error message recorded on the handle (or the last create failure when h is NULL). */
const char *ffxg_last_error(const ffxg_handle *h);

/* Copy new coordinates ([n][3], A) to the device.  ForceFieldEnergy.setCoordinates
 * (ForceFieldEnergy.java:2629). */
int ffxg_set_coordinates(ffxg_handle *h, const double *xyz);

/* A new cell: edges box[3] (A), angles[3] (alpha, beta, gamma in degrees; NULL: 90) and,
 * when pme_grid is not NULL, new PME mesh dimensions (NULL keeps the mesh, as a pme-grid
 * key does in the reference):
 * ForceFieldEnergy.setCrystal (ForceFieldEnergy.java:2650-2666), which passes the crystal to
 * ParticleMeshEwald.setCrystal (ParticleMeshEwald.java:1262-1283) and
 * ReciprocalSpace.setCrystal / initConvolution (ReciprocalSpace.java:750-761, 909-1000); the
 * FFM binding's override is OpenMMEnergy.setCrystal's counterpart (OpenMMEnergy.java:585).
 * Rebuilds the PME tables and the charge correction; the next evaluation rebuilds the
 * neighbour list and captures its graph anew.  A barostat or lattice move needs no new
 * handle. */
int ffxg_set_box(ffxg_handle *h, const double box[3], const double angles[3], const int32_t pme_grid[3]);

/* New parameter values for the same atoms, topology and vdW types: sys->multipole,
 * polarizability, thole, pdamp, red_factor, vdw_inv_rmin and vdw_eps are read (the other
 * fields are ignored; n_atoms and n_vdw_types must equal the handle's).  The counterpart
 * of OpenMMEnergy.updateParameters (OpenMMEnergy.java:623-631) for this library: a
 * parameter-fitting loop (ffxg_param_grad) updates values in place, with no allocation
 * and no new graph capture (with electrostatic lambda on, the soft atoms' vacuum
 * sub-system is rebuilt). */
int ffxg_update_parameters(ffxg_handle *h, const ffxg_system *sys);

/* Energy (and optionally gradient) at the current coordinates.
 * ForceFieldEnergy.energy(gradient, print) (ForceFieldEnergy.java:1638-1800) for the
 * vdW + PME terms.  terms[FFXG_N_TERMS] (kcal/mol), grad[n][3] (kcal/mol/A, may be
 * NULL when want_grad == 0), counts[FFXG_N_COUNTS] (may be NULL). */
int ffxg_energy(ffxg_handle *h, int want_grad, double *terms, double *grad, int64_t *counts);

/* Same as ffxg_energy with the coordinates passed in: energyAndGradient(x, g)
 * (ForceFieldEnergy.java:1843-1890) without the optimizer scaling. */
int ffxg_energy_and_gradient(ffxg_handle *h, const double *xyz, double *terms, double *grad,
                             int64_t *counts);

/* Device-resident variant used by the benchmark and by callers that keep
 * coordinates on the GPU: d_xyz[n][3] and d_grad[n][3] are device pointers on
 * the handle's device; the call is asynchronous on the handle's stream except
 * for the PCG convergence check.  terms/counts are host buffers. */
int ffxg_energy_device(ffxg_handle *h, const double *d_xyz, double *d_grad, double *terms,
                       int64_t *counts);

/* Induced dipoles from the last energy call: ParticleMeshEwald.inducedDipole[0]
 * and inducedDipoleCR[0] (ParticleMeshEwald.java:276-277), each [n][3] e*A. */
int ffxg_get_induced_dipoles(ffxg_handle *h, double *u, double *u_cr);

/* Global-frame multipoles from the last energy call ([n][10]). */
int ffxg_get_global_multipoles(ffxg_handle *h, double *mpole);

/* Cartesian reciprocal-space potential of the permanent multipoles and its first to third
 * derivatives from the last energy call, [n][20] in the tensor order t000, t100, t010,
 * t001, t200, t020, t002, t110, t101, t011, t300, t030, t003, t210, t201, t120, t021,
 * t102, t012, t111: ParticleMeshEwald.cartesianMultipolePhi (ParticleMeshEwald.java:438),
 * filled by ReciprocalSpace.computePermanentPhi (PermanentPhiLoop, ReciprocalSpace.java:
 * 2295-2454). */
int ffxg_get_permanent_potential(ffxg_handle *h, double *phi);

/* Pair set of the buffered neighbour list (NeighborList.java:905-1115) as
 * unordered (i, k) with i < k.  With pairs == NULL only *n_pairs is written. */
int ffxg_get_neighbor_pairs(ffxg_handle *h, int32_t *pairs, int64_t *n_pairs);

/* Image pairs of the buffered list, one row per image: (i, k, nx, ny, nz) with the lattice
 * shift n of x_k + n L - x_i, for k > i, or k == i and n > 0 in (z, y, x) lexicographic
 * order; n = 0 outside multi-image mode.  rows may be NULL to count. */
int ffxg_get_neighbor_images(ffxg_handle *h, int32_t *rows, int64_t *n_rows);

/* Parameter gradients of the last evaluation (the differentiation counterpart of the
 * reference's parameter fitting; it has no analytic equivalent to cite): dEdM[n][10] is
 * dE/dM of each atom's LOCAL-frame multipole in the component order of
 * ffxg_system.multipole (charge, dipole x y z, quadrupole xx yy zz xy xz yz, each
 * off-diagonal element counted once), dEdalpha[n] dE/d(polarizability) with the Thole
 * damping held fixed.  The permanent energy is bilinear in the multipoles; for
 * E_pol = -1/2 electric E_d^T A^-1 E_p with A = alpha^-1 - T symmetric, the CR dipoles
 * A^-1 E_p are the adjoint solution, so no further solve is needed.  Per-type gradients are
 * sums over the atoms of a type.  Not available under electrostatic lambda. */
int ffxg_param_grad(ffxg_handle *h, double *dEdM, double *dEdalpha);

/* Lists of every lattice image inside the cutoffs.  AUTO (the default) uses them when an
 * edge is at most twice an interaction cutoff (max of vdW, real-space and preconditioner
 * cutoffs), the boxes the reference expands into a replicate supercell
 * (ReplicatesCrystal.replicatesCrystalFactory, C/ReplicatesCrystal.java:172-202: the same
 * sum); the minimum image otherwise.  ALL forces them.  The list builder of this mode is
 * a brute-force O(N^2) pass, meant for the small boxes that need it. */
enum { FFXG_IMAGES_AUTO = 0, FFXG_IMAGES_ALL = 1 };
int ffxg_set_image_mode(ffxg_handle *h, int mode);

/* ---- Batches of independent systems --------------------------------------------------
 * Many small periodic systems of uneven size (conformer, rotamer or lambda-window
 * energies) evaluated together.  The reference evaluates such sets one ForceFieldEnergy
 * at a time (ForceFieldEnergy.energyAndGradient, P/ForceFieldEnergy.java:1843-1890, in a
 * caller's loop); here each system keeps its own handle, and one batch evaluation is one
 * CUDA graph launch.  GRAPH mode runs the batch stage by stage: each kernel of the
 * evaluation is one launch for all systems (each system a contiguous range of the grid's
 * blocks, with its own arguments), and the solver loop is one device-side loop that skips
 * the systems already converged.  BRANCHES mode replays every system's own captured
 * evaluation as a branch of one graph (GRAPH falls back to it when the systems'
 * evaluations cannot be merged into common stages); LOOP mode loops over single-system
 * launches, for comparison.  Results are those of the single-system path (bit for bit in
 * the mixed form, except a 64 x 64 mixed-form mesh, whose FFT a stage-by-stage batch
 * takes by its per-axis passes).
 *   systems[n_systems], params[n_systems]: as for ffxg_create, one per system.
 *   xyz, grad: all systems' coordinates / gradients concatenated in system order
 *     ([total atoms][3]; xyz may be NULL to reuse the last accepted coordinates;
 *     after a call rejected with FFXG_ERR_NONFINITE there are none: BAD_ARG).
 *   terms[n_systems][FFXG_N_TERMS]; counts[n_systems][FFXG_N_COUNTS] and
 *   status[n_systems] may be NULL.  Returns the first nonzero status, if any. */
typedef struct ffxg_batch ffxg_batch;
enum { FFXG_BATCH_GRAPH = 0, FFXG_BATCH_LOOP = 1, FFXG_BATCH_BRANCHES = 2 };
int ffxg_batch_create(int32_t n_systems, const ffxg_system *systems, const ffxg_params *params, ffxg_batch **out);
int ffxg_batch_energy(ffxg_batch *b, const double *xyz, int want_grad, double *terms, double *grad, int64_t *counts,
                      int32_t *status);
int ffxg_batch_set_mode(ffxg_batch *b, int mode);
/* Total atoms; offsets[n_systems + 1] (may be NULL) receives each system's first atom. */
int64_t ffxg_batch_atoms(const ffxg_batch *b, int64_t *offsets);
/* The handle of system i (induced dipoles, lambda, image mode ...); owned by the batch. */
ffxg_handle *ffxg_batch_system(ffxg_batch *b, int32_t i);
/* How many times the batch graph was captured (a new capture follows list growth or a
 * change of a system's lambda or modes). */
int64_t ffxg_batch_graph_builds(const ffxg_batch *b);
/* Stages of the batch's stage-by-stage graph for want_grad (0 when the batch has none:
 * not built yet, or BRANCHES / LOOP). */
int32_t ffxg_batch_stages(const ffxg_batch *b, int want_grad);
/* GRAPH mode runs the systems in groups of near-equal atom count, each group a branch of
 * the graph with its own stages and solver loop, so that the groups' kernels overlap.  The
 * number of groups is autotuned when the graph is first built: 1, 2, 4 and 8 groups are
 * built and timed on the device, and the fastest is kept (a batch with the ASPC predictor
 * takes 4 untimed).  ffxg_batch_tuning returns the chosen number (0 before the first
 * build) and fills candidates[4] / ms[4] (each may be NULL) with the candidates timed and
 * their milliseconds per batch; ffxg_batch_set_groups fixes the number instead (0: tune
 * again) and drops the built graphs. */
int32_t ffxg_batch_tuning(const ffxg_batch *b, int32_t *candidates, double *ms);
int ffxg_batch_set_groups(ffxg_batch *b, int32_t groups);
const char *ffxg_batch_last_error(const ffxg_batch *b);
void ffxg_batch_destroy(ffxg_batch *b);

/* Alchemical state of the van der Waals term: which atoms carry lambda (Atom.applyLambda)
 * and the softcore keys read by VanDerWaals (VanDerWaals.java:336-357).  soft[n] is
 * 0/1; molecule[n] (may be NULL: every atom its own molecule) decides the both-soft
 * intermolecular / intramolecular softcore options.  Defaults of the reference:
 * vdw-lambda-alpha 0.25, vdw-lambda-exponent 3, vdw-lambda-end 1, both options off.
 * A pair is softcore when exactly one atom is soft (or both, per the options); its
 * energy is eps * L^n * t1 * t2 with alpha (1 - L)^2 added to both denominators
 * (VanDerWaalsLoop, VanDerWaals.java:1723-1880).
 *
 * elec != 0 also decouples the soft atoms' electrostatics as the reference's
 * elec-lambdaterm in OST mode (ParticleMeshEwald.java:897-935, 1609-1796): the energy is
 * the sum of (1) the whole system with softcore permanent real-space pairs involving a
 * soft atom (r^2 + alpha (1 - L_p)^2, scaled by L_p^n), permanent reciprocal space scaled
 * by L_p^n and polarization scaled by the polarization window's power; (2) the system
 * without the soft atoms, reciprocal permanent and polarization scaled by the
 * complements; (3) the soft atoms alone in vacuum (no Ewald, no cutoff), scaled by the
 * complements.  L_p is lambda mapped into [permanent_lambda_start, _end], the
 * polarization window likewise (AlchemicalParameters.update, pme/AlchemicalParameters.
 * java:306-380).  Reference defaults: permanent-lambda-alpha 2, -exponent 3, -start 0.4,
 * -end 1; polarization-lambda-start 0.75, -end 1, -exponent 3; ligand-vapor-elec and
 * no-ligand-condensed-scf on.  The vacuum step solves its dipoles with the same PCG as
 * the periodic steps (the reference uses SOR there): the two agree to the SCF
 * tolerance. */
typedef struct ffxg_alchemy {
  const int32_t *soft;
  const int32_t *molecule;
  double vdw_lambda_alpha;
  double vdw_lambda_exponent;
  double vdw_lambda_end;
  int32_t intermolecular_softcore;
  int32_t intramolecular_softcore;
  int32_t elec;
  double permanent_lambda_alpha;
  double permanent_lambda_exponent;
  double permanent_lambda_start;
  double permanent_lambda_end;
  double polarization_lambda_start;
  double polarization_lambda_end;
  double polarization_lambda_exponent;
  int32_t ligand_vapor_elec;
  int32_t no_ligand_condensed_scf;
} ffxg_alchemy;

/* Set (or, with a == NULL, clear) the soft atoms and softcore keys.  The state starts
 * cleared and lambda at 1. */
int ffxg_set_alchemy(ffxg_handle *h, const ffxg_alchemy *a);

/* LambdaInterface.setLambda (P/bonded/LambdaInterface.java:47-99) for the vdW term:
 * lambda in [0, 1], rescaled by vdw-lambda-end as VanDerWaals.setLambda (:599-647). */
int ffxg_set_lambda(ffxg_handle *h, double lambda);

/* dU/dL, d2U/dL2 and dU/dX dL (LambdaInterface getdEdL / getd2EdL2 / getdEdXdL) of the
 * last evaluation: the vdW softcore contributions, plus the electrostatic ones with
 * elec set.  dEdXdL[n][3] (may be NULL) is filled
 * only when that evaluation computed a gradient. */
int ffxg_get_dEdL(ffxg_handle *h, double *dEdL, double *d2EdL2, double *dEdXdL);

/* Molecular dynamics on the device: VelocityVerlet (algorithms/.../integrators/
 * VelocityVerlet.java:73-120) with SettleConstraint rigid three-site molecules
 * (P/constraint/SettleConstraint.java), the counterpart of MolecularDynamics.mainLoop
 * (MolecularDynamics.java:1488-1560) for this library's vdW + PME potential.  mass[n]
 * in amu (0 freezes an atom); settle[n_settle][3] lists each rigid molecule as its
 * centre atom and two partners at distance settle_d1 from the centre and settle_d2 from
 * each other (water: O, H, H; 0.9572 A and 1.5139 A for 104.52 degrees). */
typedef struct ffxg_md {
  const double *mass;
  int32_t n_settle;
  const int32_t *settle;
  double settle_d1;
  double settle_d2;
} ffxg_md;
int ffxg_md_setup(ffxg_handle *h, const ffxg_md *md);

/* Integrate n_steps of dt (ps) from xyz[n][3] (A) and vel[n][3] (A/ps), both updated in
 * place.  Forces are this library's energy gradient; units follow the reference
 * (a = -418.4 g / m).  epot[n_steps] and ekin[n_steps] (kcal/mol, may be NULL) receive
 * the potential energy after each step's force evaluation and the kinetic energy after
 * its closing half kick.  Positions and velocities stay on the device between steps. */
int ffxg_md_run(ffxg_handle *h, double dt, int32_t n_steps, double *xyz, double *vel, double *epot, double *ekin);

/* SCF predictor for the PCG starting guess (the scf-predictor key, ParticleMeshEwald.java:
 * 540-550): FFXG_PREDICTOR_ASPC is the always-stable predictor of
 * SCFPredictorParameters.aspcPredictor (pme/SCFPredictorParameters.java:80-123), which
 * starts each solve from the direct dipoles plus a fixed combination of the last six
 * converged (u - u_direct); it applies once six solves are stored and leaves the
 * converged result unchanged up to polar-eps.  Setting a predictor clears the history. */
enum { FFXG_PREDICTOR_NONE = 0, FFXG_PREDICTOR_ASPC = 1 };
int ffxg_set_scf_predictor(ffxg_handle *h, int predictor);

/* The CUDA stream (cudaStream_t) the handle launches on, for event timing. */
void *ffxg_stream(ffxg_handle *h);

/* Neighbour-list builds since the handle was created (every evaluation and MD step that
 * found an atom moved more than half the list buffer, as NeighborList's motion check
 * decides, NeighborList.java:777-799), for MD statistics. */
int64_t ffxg_list_builds(const ffxg_handle *h);

/* Device count of kernel launches issued by the last energy call. */
int64_t ffxg_last_launch_count(const ffxg_handle *h);

/* Per-stage device timings, the counterpart of PMETimings (pme/PMETimings.java:60-124)
 * and the per-thread vdW / neighbour-list timers (VanDerWaals.java:1241-1288).  With
 * timing on, every stage launch is bracketed by CUDA events on the handle's stream;
 * ffxg_get_timings returns the accumulated milliseconds and launch counts per stage
 * since timing was (re)enabled. */
enum {
  FFXG_STAGE_LISTS = 0,          /* coordinates, motion check, cell and Verlet lists */
  FFXG_STAGE_VDW = 1,
  FFXG_STAGE_MULTIPOLES = 2,     /* rotation, B-splines, fractional multipoles */
  FFXG_STAGE_PERM_RECIP = 3,     /* permanent spread + FFT convolution + potential */
  FFXG_STAGE_PERM_FIELD = 4,     /* real-space permanent field + direct dipoles */
  FFXG_STAGE_IND_RECIP = 5,      /* induced spread + FFT convolution + potential */
  FFXG_STAGE_IND_FIELD = 6,      /* real-space induced field (one launch per field) */
  FFXG_STAGE_PRECOND = 7,        /* preconditioner field */
  FFXG_STAGE_PCG_VECTOR = 8,     /* PCG vector updates and dot products */
  FFXG_STAGE_REAL_ENERGY = 9,    /* real-space energy, force and torque */
  FFXG_STAGE_RECIP_ENERGY = 10,  /* reciprocal-space energy, force and torque */
  FFXG_STAGE_GRADIENT = 11,      /* torque to gradient, assembly, sums */
  FFXG_N_STAGES = 12
};
int ffxg_set_timing(ffxg_handle *h, int on);
int ffxg_get_timings(ffxg_handle *h, double *ms, int64_t *launches, int n);

/* Execution mode (no counterpart in the reference, which has no GPU path).  With graph
 * mode on (the default) the first evaluation after the neighbour list exists captures
 * the whole evaluation, the PCG loop included as a conditional while node that the
 * solver re-arms on the device, and later evaluations replay it with one launch and
 * one synchronisation.  Off: every kernel is launched directly and the host reads the
 * solver's stopping decision after each iteration.  Results are the same either way;
 * stage timing (ffxg_set_timing) always uses direct launches. */
int ffxg_set_graph_mode(ffxg_handle *h, int on);

/* Permanent-multipole reciprocal-space potential and energy without any device
 * allocation.  This entry point has no counterpart in the reference; it is for
 * callers that may not allocate device memory themselves or through this library:
 * a process whose GPU memory is owned by another allocator (a framework's caching
 * pool, a JVM or plugin host that forbids new device allocations after start-up),
 * or a latency-critical caller that must not pay cudaMalloc's implicit
 * synchronisation.  It creates no handle and calls no allocator.
 *
 * Inputs and outputs are the caller's device buffers on the current device:
 * d_xyz[n][3] coordinates (A), d_mpole[n][10] global-frame multipoles (the order of
 * ffxg_get_global_multipoles), d_phi[n][10] Cartesian potential and derivatives
 * (may be NULL) and d_energy[1], the permanent reciprocal energy 1/2 * electric *
 * sum(M . Phi) (kcal/mol, the FFXG_TERM_PERM_RECIP of a neutral cell).  box[3] and
 * pme_grid[3] are host arrays; `stream` is a cudaStream_t (NULL: the legacy default
 * stream) and the call is asynchronous on it.
 *
 * All intermediates live in one fixed array of about 6.3 MB that each device
 * holds from the first call until the process exits.  Limits: n_atoms <= 32768 and
 * every mesh dimension <= 64 (and >= 5, any factors); beyond them the call returns
 * FFXG_ERR_CAPACITY without launching anything.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  Every call on a device shares
 * the one array: calls that overlap on the GPU (different streams or threads)
 * race, so the caller must serialise them.  Each call clears the mesh itself. */
int ffxg_pme_recip_permanent_noalloc(const double *d_xyz, const double *d_mpole, int32_t n_atoms,
                                     const double box[3], const int32_t pme_grid[3], double ewald_alpha,
                                     double electric, double *d_phi, double *d_energy, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FFXCUDA_H */
