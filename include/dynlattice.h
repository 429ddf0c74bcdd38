/*
 * dynlattice.h -- C ABI of the B200 explicit-dynamics engine for
 * geometrically exact (Simo--Reissner / Simo--Vu-Quoc) Cosserat rod lattices.
 *
 * The engine replaces the explicit path of dynLattice, which is a set of JIVE
 * plugins behind string-dispatched `takeAction` calls:
 *
 *   ModelFactory "specialCosseratRod"  src/models/SpecialCosseratRodModel.cpp:1218-1223
 *   ModelFactory "Lattice"             src/models/LatticeModel.cpp:334-337
 *   ModelFactory "RodContact"          src/models/RodContactModel.cpp:1226-1231
 *   ModelFactory "JointContact"        src/models/JointContactModel.cpp:352
 *   ModelFactory "Mass"                src/models/MassModel.cpp:137-138
 *   MaterialFactory "ElasticRod"       src/materials/ElasticRodMaterial.cpp:420-424
 *   MaterialFactory "ElastoPlasticRod" src/materials/ElastoPlasticRodMaterial.cpp:388-392
 *   ModuleFactory "LeapFrog"           src/modules/LeapFrogModule.cpp:105-110
 *   ModuleFactory "MilneDevice"        src/modules/MilneDeviceModule.cpp:165
 *   ModuleFactory "GroupOutput", "CSVOutput", "ParaView" (output of a .pro run)
 *                                      src/modules/GroupOutputModule.cpp:219,
 *                                      CSVOutputModule.cpp:68-69, ParaViewModule.cpp:705
 *
 * Conventions: every call returns an int status (DL_OK == 0); no C++
 * exception crosses this boundary; a failed call leaves a message that
 * dl_last_error() returns (per thread).  Host buffers are owned by the
 * caller; device buffers are owned by the engine.  One handle must be used by
 * one host thread at a time.  All device work of a handle runs on the CUDA
 * stream given to dl_set_stream (default: the legacy default stream).
 *
 * DOF order per node everywhere: (dx, dy, dz, rx, ry, rz) -- translations
 * first, then rotations, as SpecialCosseratRodModel's TRANS_PART/ROT_PART
 * (src/models/SpecialCosseratRodModel.cpp:40-41).
 */
#ifndef DYNLATTICE_H
#define DYNLATTICE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#define DL_EXTERN extern "C"
#else
#define DL_EXTERN extern
#endif
#define DL_API DL_EXTERN __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* status codes                                                        */
/* ------------------------------------------------------------------ */
enum dl_status {
  DL_OK = 0,
  DL_ERR_INVALID = 1,      /* bad argument or inconsistent model            */
  DL_ERR_CUDA = 2,         /* a CUDA runtime call failed                    */
  DL_ERR_PARSE = 3,        /* .pro / expression / mesh syntax error         */
  DL_ERR_RETURN_MAP = 4,   /* return map hit maxIter (reference: JEM_PRECHECK2
                              "Too many iterations in plasticity loop",
                              ElastoPlasticRodMaterial.cpp:234)             */
  DL_ERR_NONFINITE = 5,    /* NaN/Inf in the state                          */
  DL_ERR_MASS = 6,         /* zero or negative mass (ExplicitModule.cpp:452) */
  DL_ERR_TIMEOUT = 7,      /* a bounded device wait gave up                 */
  DL_ERR_UNSUPPORTED = 8,  /* feature outside the engine's subset           */
  DL_ERR_IO = 9,           /* file could not be read/written                */
  DL_ERR_NOMEM = 10,       /* device or host allocation failed              */
  DL_ERR_NO_DEVICE = 11,   /* no CUDA device: the engine has no CPU path    */
  DL_ERR_CONTACT = 12      /* contact candidate list went stale: raise the
                              margin (dl_contact_desc.margin)               */
};

/* device error word bits (dl_get_error_word) */
#define DL_EW_RETURN_MAP 0x1u
#define DL_EW_NONFINITE  0x2u
#define DL_EW_TIMEOUT    0x4u
#define DL_EW_MASS       0x8u
#define DL_EW_CONTACT_OVERFLOW 0x10u
#define DL_EW_CONTACT_STALE    0x20u  /* a node moved more than half the
                                          candidate-list margin between two
                                          list rebuilds: pairs may be missing */
#define DL_EW_STEP_CONTROL     0x40u  /* MilneDevice: non-finite error estimate,
                                          or a step still rejected after 1000
                                          attempts */

/* precision of the element force / return map; state is always FP64 */
enum dl_precision { DL_PLAIN_FP64 = 0, DL_MIXED = 1 };

/* material types (MaterialFactory names) */
enum dl_material_type { DL_MAT_ELASTIC_ROD = 0, DL_MAT_ELASTOPLASTIC_ROD = 1 };

/* boundary-condition kinds */
enum dl_bc_kind {
  DL_BC_DIRICHLET = 0,  /* prescribed ACCELERATION of a DOF (explicit runs constrain
                           accelerations: ExplicitModule.cpp:352-356)          */
  DL_BC_NEUMANN = 1,    /* nodal force/moment (NeumannModel.cpp:291-348)      */
  DL_BC_INIT_VELO = 2,  /* initial velocity (InitLoadModel.cpp:95-137)         */
  DL_BC_INIT_DISP = 3,  /* initial displacement of a translational DOF         */
  DL_BC_MASS = 4        /* added point mass: factor is added to the diagonal of
                           the node's mass matrix for this DOF (MassModel,
                           MassModel.cpp:77-99: totalMass / group size)        */
};

/* ------------------------------------------------------------------ */
/* model description: plain arrays, caller-owned, read during create   */
/* ------------------------------------------------------------------ */

/* One material (ElasticRodMaterial / ElastoPlasticRodMaterial keys,
 * ElasticRodMaterial.cpp:32-46,65-207; ElastoPlasticRodMaterial.cpp:31-35,55-146). */
typedef struct dl_material_desc {
  int32_t type;               /* dl_material_type                               */
  double young;               /* "young"                                        */
  double shear_modulus;       /* "shear_modulus" (or young/2/(1+nu))            */
  double shear_correction;    /* "shear_correction" (circle 0.9, else 5/6)      */
  double area;                /* section area                                   */
  double area_moment[2];      /* I1, I2                                         */
  double polar_moment;        /* J (default I1+I2)                              */
  double density;             /* "density"                                      */
  double inertia_correct;     /* "inertia_correct" factor on rotational mass (1) */
  int32_t circle;             /* 1: circular section -- enables the per-element
                                 radius override in dl_model_desc.elem_radius     */
  double radius;              /* circle radius                                  */
  /* elastoplastic part */
  const char *yield_cond;     /* "yieldCond" expression                         */
  const char *const *yield_deriv; /* "yieldDeriv" expressions (may be NULL)     */
  int32_t n_yield_deriv;      /* 0, or 6 + hardening count                      */
  int32_t has_isotropic;      /* "isotropicCoefficient" present                 */
  double isotropic_coefficient;
  const double *kinematic_tensor; /* "kinematicTensor" 36 values or NULL        */
  int32_t max_iter;           /* "maxIter" (20)                                 */
  double precision;           /* "precision" (1e-5)                             */
} dl_material_desc;

typedef struct dl_bc_desc {
  int32_t kind;               /* dl_bc_kind                                     */
  int32_t dof;                /* 0..5                                           */
  int32_t n_nodes;
  const int32_t *nodes;       /* node indices                                   */
  double factor;              /* "factors" entry                                */
  const char *scale;          /* scale expression in t, i, deltaTime; NULL = 1.
                                 Dirichlet INCREMENT method becomes
                                 "initDisp + (i-1)*dispIncr" (DirichletModel.cpp:184-205,265-282) */
} dl_bc_desc;

/* Rigid plate (engine extension, not a reference feature): node--plane
 * penalty.  A node at x penetrates when g = (x - p(t)).n - radius < 0 with
 * p(t) = point0 + velocity t; its internal force gets penalty * g * n. */
typedef struct dl_plate_desc {
  double normal[3];           /* unit normal pointing into the lattice         */
  double point0[3];           /* a point of the plate at t = 0                 */
  double velocity[3];         /* plate velocity                                */
  double penalty;             /* penalty stiffness per unit penetration        */
} dl_plate_desc;

/* Rod--rod penalty contact (RodContactModel.cpp:24-97) */
typedef struct dl_contact_desc {
  int32_t enabled;
  double radius;              /* contact radius r: active when distance <= 2r  */
  double penalty_sts;         /* "penaltySTS" (or "penalty")                    */
  double penalty_nts;         /* "penaltyNTS" (or "penalty")                    */
  double margin;              /* candidate-list margin (engine): 0 = radius/2  */
  int32_t max_pairs;          /* capacity of the candidate list; 0 = automatic  */
  int32_t n_plates;           /* 0..2 rigid plates                             */
  dl_plate_desc plates[2];
} dl_contact_desc;

/* Joint contact ("jointContact" of the Lattice model, LatticeModel.cpp:99-101;
 * JointContactModel.cpp:24-97, 236-353).  The joints are the nodes of the
 * element group "points" (the mesh's point elements).  Two joints A, B (A
 * before B in the list) interact when their distance d is at most 2r now and
 * their reference distance is more than 2r; then, with n = (x_B - x_A) / d,
 *   f_int(A) -= penalty (2r - d) n,   f_int(B) += penalty (2r - d) n
 * (translational DOFs only), which with f_res = f_ext - f_int pulls the two
 * joints together.  Joints at d = 0 get no force (the reference's normal is
 * undefined there). */
typedef struct dl_joint_contact_desc {
  int32_t enabled;
  double radius;              /* joint radius r                                 */
  double penalty;             /* "penalty"                                      */
  int32_t n_joints;
  const int32_t *joints;      /* node indices, in the order of the "points" group */
  double margin;              /* candidate-list margin (engine): 0 = radius/2  */
} dl_joint_contact_desc;

typedef struct dl_model_desc {
  int32_t n_nodes;
  const double *coords;       /* [n_nodes][3] reference positions X0            */
  int32_t n_elems;
  int32_t nodes_per_elem;     /* 2, 3 or 4 (Line2/3/4; contact, batches and the
                                 adjoint take 2)                                  */
  const int32_t *conn;        /* [n_elems][nodes_per_elem], nodes along the line */
  const int32_t *elem_rod;    /* [n_elems] rod (element group "beam_k") index;
                                 elements of one rod in mesh order            */
  int32_t n_rods;
  const int32_t *elem_mat;    /* [n_elems] material index, NULL = all 0        */
  const double *elem_radius;  /* [n_elems] per-element circle radius, or NULL   */
  int32_t n_materials;
  const dl_material_desc *materials;
  const char *const *dof_names; /* 6 names used by expressions; NULL = dx..rz   */
  int32_t n_gauss;            /* Gauss points per element (stiffShape.intScheme) */
  int32_t has_material_ey;    /* "material_ey" given                            */
  double material_ey[3];
  /* per-node tangent overrides ("given_dir_nodes"/"given_dir_dirs"), applied to
     every rod containing the node; may be NULL */
  int32_t n_given_dirs;
  const int32_t *given_dir_nodes;
  const double *given_dirs;   /* [n_given_dirs][3] */
  int32_t n_bcs;
  const dl_bc_desc *bcs;
  double dt;                  /* "deltaTime"                                    */
  int32_t so3_update;         /* 1: exponential-map rotation update ("dofs_SO3")*/
  int32_t gyroscopic;         /* 1: add omega x (Theta omega) to the internal force */
  dl_contact_desc contact;
  dl_joint_contact_desc joint_contact;
  /* mass matrix of the explicit module (ExplicitModule.cpp:154-172):
     DL_MASS_CONSISTENT (0, default) solves each node's 6x6 block with the
     gyroscopic term; DL_MASS_LUMPED (1) keeps the diagonal of that block
     (the model's MATRIX2 assembled into a diagonal matrix, a = M^-1 r per
     DOF, ExplicitModule.cpp:339-357, 445-453) and drops the gyroscopic
     term, which the rod model adds only when it is given the consistent
     matrix (SpecialCosseratRodModel.cpp:351-355) */
  int32_t mass_mode;
  /* rigid ties (HingeModel "rigidHinge", HingeModel.cpp:93-105, 172-199):
     ties[2k] is a master node, ties[2k+1] a slave that shares all six of its
     DOFs; a slave has one master and a master is no slave.  In an explicit
     run the hinge's plastic offset stays zero (it changes only in
     CHECK_COMMIT, which the explicit modules never issue), and the
     consistent solve condenses the constraint: each group moves as one node
     with the summed mass, forces and boundary conditions of its members.
     The lumped mode's setSlaveDofs rule is not provided (refused). */
  int32_t n_ties;
  const int32_t *ties;
} dl_model_desc;

enum { DL_MASS_CONSISTENT = 0, DL_MASS_LUMPED = 1 };

/* One sampled record: per watched node x(3) theta(3) v(6), then energies. */
typedef struct dl_energies {
  double kinetic;             /* 1/2 v^T M v            (LatticeModel.cpp:223-250)   */
  double potential;           /* sum w 1/2 eps_e.sigma  (SpecialCosseratRodModel.cpp:1074-1107) */
  double dissipated;          /* accumulated plastic work (ElastoPlasticRodMaterial.cpp:271-307) */
  double external_work;       /* work of Neumann loads (engine extension)      */
  double contact;             /* penalty energy of active contacts (extension) */
} dl_energies;

typedef struct dl_handle_s dl_handle;

/* ------------------------------------------------------------------ */
/* lifetime                                                            */
/* ------------------------------------------------------------------ */

/* Last error message of the calling thread ("" if none). */
DL_API const char *dl_last_error(void);

/* ------------------------------------------------------------------ */
/* time integrator                                                     */
/* ------------------------------------------------------------------ */

enum { DL_INTEG_LEAPFROG = 0, DL_INTEG_MILNE = 1 };

/* Explicit integrator of a single lattice (ModuleFactory "LeapFrog" /
 * "MilneDevice", ExplicitModule.cpp:23-26, 60-148).  LeapFrog (default):
 * fixed dt.  MilneDevice: order-1 predictor-corrector with two force
 * evaluations per step (MilneDeviceModule::solve, MilneDeviceModule.cpp:41-118)
 * and error-controlled dt (ExplicitModule::commit, ExplicitModule.cpp:291-334):
 *   error = (q(u_pre, u_new) + dt q(v_pre, v_new)) / 2,
 *   q(a, b) = ||(a - b) with translations / length_scale||_2 / sqrt(6 n_nodes),
 *   dt_opt = dt sqrt(precision / error);
 *   accepted (error <= precision or dt <= min_dt):
 *     dt = max(min(safety dt_opt, increase dt, max_dt), decrease dt, min_dt)
 *   rejected: dt = max(safety dt_opt, decrease dt, min_dt), step repeated.
 * dl_run(h, n) then advances n ACCEPTED steps.  Zero fields take the
 * reference defaults: min_dt = dt0/100, max_dt = 100 dt0, safety 0.9,
 * increase 1.2, decrease 0.8, length_scale 1e-3; precision has no default
 * here (the reference inherits jive::solver::Solver::PRECISION, whose value
 * the absent JIVE headers would give) and must be > 0 for MilneDevice.
 * MilneDevice runs single lattices without contact or plates, in the
 * persistent launch; time-dependent load scales are evaluated on the device
 * at the adapted times. */
typedef struct {
  int32_t kind;            /* DL_INTEG_LEAPFROG or DL_INTEG_MILNE */
  double precision;        /* "precision" */
  double min_dt, max_dt;   /* minimum / maximum time step (0: defaults) */
  double safety;           /* "stepSaftey" */
  double increase;         /* "increaseFactor" */
  double decrease;         /* "decreaseFactor" */
  double length_scale;     /* "lengthScale" */
} dl_integrator_desc;

/* Number of CUDA devices visible (0 on a machine without a GPU). */
DL_API int dl_device_count(int *count);

/* Build an engine from a model description.  Replaces the JIVE INIT action of
 * LatticeModel/SpecialCosseratRodModel/ExplicitModule:
 *   SpecialCosseratRodModel::initRotation_ (SpecialCosseratRodModel.cpp:574-658),
 *   ::initStrain_ (:536-569), ExplicitModule::init (ExplicitModule.cpp:58-196). */
DL_API int dl_create(const dl_model_desc *desc, int precision, dl_handle **out);

/* Build an engine from a dynLattice .pro file, meshing the .geo/.msh it names
 * (dl_pro_open + dl_create).  Replaces the reference's input chain
 * GMSHInputModule (GMSHInputModule.cpp:137-415), GroupInputModule
 * (GroupInputModule.cpp:165-500) and the model/module configure() calls. */
DL_API int dl_create_from_pro(const char *pro_path, int precision, dl_handle **out);

/* The parsed input of a .pro file: model description (valid until
 * dl_pro_close), run length from control.runWhile (-1 when absent) and node
 * groups (GroupInput groups, "all", and the nodes of each line group
 * "beam_k"). */
typedef struct dl_pro_s dl_pro;
DL_API int dl_pro_open(const char *pro_path, dl_pro **out);
DL_API int dl_pro_desc(dl_pro *p, const dl_model_desc **desc);
DL_API int dl_pro_steps(dl_pro *p, int64_t *nsteps);
DL_API int dl_pro_group(dl_pro *p, const char *name, int32_t *n_nodes, const int32_t **nodes);
/* The explicit module of the .pro file (Solver.integrator: type, deltaTime,
 * precision, minDtime, maxDtime, stepSaftey, increaseFactor, decreaseFactor,
 * lengthScale); dl_create_from_pro applies it. */
DL_API int dl_pro_integrator(dl_pro *p, dl_integrator_desc *out);
/* End time of a time-based control.runWhile ("t < T", "t <= T"), -1 when
 * the run length is given in steps or not at all (MilneDevice runs advance
 * until this time). */
DL_API int dl_pro_end_time(dl_pro *p, double *t_end);
/* Properties the file sets that the engine reads but does not apply (an
 * explicit-module updateWhen other than the default, ParaView node tables
 * other than fint/fext/fres, models of other types, ...): *n receives their
 * count; note i (0 <= i < *n) is returned through *text when text is not NULL
 * (valid until dl_pro_close). */
DL_API int dl_pro_note(dl_pro *p, int32_t i, int32_t *n, const char **text);

/* Run the .pro file's control loop on h (created from the same file) with
 * its output modules, until control.runWhile ends or max_steps steps
 * (< 0: no cap): GroupOutput (group sums of load and internal force, group
 * means of displacement and velocity as variables <group>.<load|resp|disp|
 * velo>.<dof>, GroupOutputModule.cpp:70-166), Sample (dataSets expressions
 * over t, i, deltaTime, runtime, kineticEnergy, potentialEnergy,
 * dissipatedEnergy, externalWork and the group variables, one row per step
 * where sampleWhen holds, gzip when the file ends in .gz), CSVOutput
 * ("state|velo = <label>" vectors with a "time,label,<dof>[<node>]" header,
 * CSVDataPrinter.cpp:84-227) and ParaView (dl_write_vtu files named by
 * output_format with %i the output counter, plus the .pvd collection).
 * Output paths are relative to out_dir.  Conditions that use only t, i and
 * deltaTime let a LeapFrog run advance to the next output step in one
 * dl_run; otherwise, and with MilneDevice, the loop advances step by step. */
DL_API int dl_pro_run(dl_pro *p, dl_handle *h, const char *out_dir, int64_t max_steps, int64_t *steps_run);

/* ParaView output of the current state (ParaViewModule::writeFile_ /
 * writePiece_, ParaViewModule.cpp:236-620): an ASCII UnstructuredGrid of the
 * reference coordinates and Line2 cells with the point data Displacement,
 * Velocity, otherDofsDisp (rotation vector), otherDofsVelo (angular
 * velocity) and, by the flags in node_data, the internal (1), external (2)
 * and resulting (4) forces and torques.  A .pro file's ParaView module
 * (dl_pro_run) also writes its element tables (el_data) as cell data. */
DL_API int dl_write_vtu(dl_handle *h, const char *path, int32_t node_data);

/* Element table at the current state, out[n_elems][6] in the caller's element
 * numbering: the reference's GET_TABLE for elements as ParaViewModule writes
 * it (SpecialCosseratRodModel.cpp:233-248, 426-532; ParaViewModule.cpp:
 * 585-616).  name: "strain" / "mat_strain" (Gamma - Gamma0, K - K0, spatial or
 * material frame), "stress" / "mat_stress" (n, m = C (eps - eps_p) with the
 * committed plastic strain, as for the output load case), "plast_strain"
 * (committed plastic strain; zeros for elastic materials).  Per element the
 * Gauss points' values are summed and the sum is multiplied by the point
 * count: ParaViewModule scales the table rows by the accumulated weights
 * without inverting them (ParaViewModule.cpp:612). */
DL_API int dl_element_table(dl_handle *h, const char *name, double *out);

/* ParaView .pvd collection of n files with their times. */
DL_API int dl_write_pvd(const char *path, int32_t n, const double *times, const char *const *files);
DL_API int dl_pro_close(dl_pro *p);

DL_API int dl_destroy(dl_handle *h);

/* Use this CUDA stream (cudaStream_t passed as void*) for all device work. */
DL_API int dl_set_stream(dl_handle *h, void *stream);

/* ------------------------------------------------------------------ */
/* stepping                                                            */
/* ------------------------------------------------------------------ */

/* Execution mode of dl_run: 0 = one persistent cooperative launch per call
 * (element and node phases separated by a bounded grid barrier), 1 = two
 * kernel launches per step, 2 = as 0, captured once per block length as a
 * CUDA graph and replayed with updated kernel arguments. */
DL_API int dl_set_exec_mode(dl_handle *h, int mode);

/* Autotuner (engine extension): times dl_run calls of `steps` steps (at
 * least 50 steps in all) on a fresh copy of the lattice for each launch shape
 * (persistent launch with 256/128/64/32 threads per block, two launches per
 * step) and keeps the fastest for this handle.  Outputs (optional): the
 * chosen mode, threads per block (0 = per-step kernels) and its time per call
 * in ms. */
DL_API int dl_autotune(dl_handle *h, int64_t steps, int32_t *best_mode,
                       int32_t *best_threads, double *best_ms);

/* Threads per block of the persistent launch: 0 = automatic (256, halved
 * while the grid would not cover every SM), or 32/64/128/256. */
DL_API int dl_set_threads(dl_handle *h, int32_t threads);

/* Advance nsteps explicit steps (LeapFrogModule::solve, LeapFrogModule.cpp:44-84,
 * with ExplicitModule::getForce/getAcce/updateVec, ExplicitModule.cpp:339-419).
 * Asynchronous on the handle's stream: returns after enqueueing; device-side
 * failures (return map, non-finite state, barrier timeout) are reported by
 * the next dl_synchronize. */
DL_API int dl_run(dl_handle *h, int64_t nsteps);

/* Select the integrator (see dl_integrator_desc); LeapFrog until called. */
DL_API int dl_set_integrator(dl_handle *h, const dl_integrator_desc *d);

/* Time, current time step, accepted step count and rejected attempts
 * (MilneDevice; 0 for LeapFrog).  Synchronises the handle's stream. */
DL_API int dl_get_time(dl_handle *h, double *t, double *dt, int64_t *step,
                       int64_t *rejected);

/* Time of each recorded sample (the steps of dl_get_samples). */
DL_API int dl_get_sample_times(dl_handle *h, double *times, int64_t max_samples);

/* Which kernel variant runs: jit_active = 1 when the elastoplastic yield
 * function was compiled into the step kernels at create time (NVRTC, sm_100a),
 * 0 for the ahead-of-time kernels (elastic lattices, or the interpreted yield
 * program when runtime compilation is unavailable: then *jit_log says why).
 * persistent_blocks = CTAs of the persistent launch. */
DL_API int dl_get_info(dl_handle *h, int32_t *jit_active, int32_t *persistent_blocks,
                       const char **jit_log);

/* Record samples every `every` steps of the following dl_run calls: for each
 * watched node x, theta, v and the energies.  n_watch may be 0.
 * Replaces the Sample / GroupOutput modules' per-step reads
 * (GroupOutputModule.cpp:70-190). */
DL_API int dl_set_sampling(dl_handle *h, int32_t every, int32_t n_watch,
                           const int32_t *watch_nodes, int64_t capacity);
/* Copy recorded samples to host: steps[s]; node_rows[s][watch][12] =
 * u(3), theta(3), v(6) per watched node; one dl_energies per sample. */
DL_API int dl_get_samples(dl_handle *h, int64_t *n_samples, int64_t *steps,
                          double *node_rows, dl_energies *energies,
                          int64_t max_samples);

/* Clear the handle's error word (the device-side failure flags that
 * dl_synchronize reports) and reset its grid barrier, so that the handle can
 * run again after a reported failure; the state is the one the failed run
 * left (set it again with dl_set_state where that matters).  Engine feature:
 * the reference aborts the run with an exception instead (return map,
 * ElastoPlasticRodMaterial.cpp:234; zero masses, ExplicitModule.cpp:450-453). */
DL_API int dl_clear_error(dl_handle *h);

/* Failure-path hook of the tests: bound one grid-barrier wait at limit_us
 * microseconds (0: about 2 s) and make the barrier expect phantom_blocks (0
 * or 1) blocks beyond the launch's own, which never arrive, so that every
 * wait runs out, the kernel returns and dl_synchronize reports
 * DL_ERR_TIMEOUT.  No counterpart in the reference. */
DL_API int dl_set_barrier_test(dl_handle *h, uint32_t limit_us, uint32_t phantom_blocks);

/* Synchronise the handle's stream, then read the device error word. */
DL_API int dl_get_error_word(dl_handle *h, uint32_t *word);

/* Wait for the handle's stream; returns the status of the device error word. */
DL_API int dl_synchronize(dl_handle *h);

/* ------------------------------------------------------------------ */
/* state access (host buffers, synchronous)                            */
/* ------------------------------------------------------------------ */

DL_API int dl_get_sizes(dl_handle *h, int32_t *n_nodes, int32_t *n_elems,
                        int32_t *n_gauss, int64_t *step);

/* u: [n_nodes][3] displacement; theta: [n_nodes][3] total rotation vector
 * log(R) as the reference's rx,ry,rz DOFs; v: [n_nodes][6]. Any may be NULL. */
DL_API int dl_get_state(dl_handle *h, double *u, double *theta, double *v);
DL_API int dl_set_state(dl_handle *h, const double *u, const double *theta,
                        const double *v);

/* Energies after the last step (definitions as in dl_energies). */
DL_API int dl_get_energies(dl_handle *h, dl_energies *e);

/* Internal force vector of a given configuration without advancing:
 * fint [n_nodes][6] (GET_INT_VECTOR, SpecialCosseratRodModel.cpp:330-365;
 * no history update; gyroscopic term excluded). */
DL_API int dl_internal_force(dl_handle *h, const double *u, const double *theta,
                             double *fint);

/* Allocation-free variant of dl_internal_force for callers that cannot
 * allocate device memory when they need the force: a real-time loop with a
 * fixed memory budget (a cudaMalloc there may synchronise the device and miss
 * the loop's deadline), or a host framework that owns all device allocations
 * and forbids new ones once it runs.  No counterpart in the reference.
 * u_dev/theta_dev [n_nodes][3] and fint_dev [n_nodes][6] are DEVICE arrays on
 * the handle's device (the device current at dl_create), in the caller's node
 * numbering; the call makes that device current while it runs and restores
 * the caller's device.  Scratch memory is one static device array of 24 MiB
 * per GPU (held from library load to process exit); lattices needing more
 * (2*r(32 n_nodes) + r(12 n_elems sizeof(element precision)) bytes, r = round
 * up to 256) are rejected with DL_ERR_INVALID.  The first call on a device
 * resolves the array's device address (cudaGetSymbolAddress): make that first
 * call before any stream capture.  All calls share the array; calls whose GPU
 * work overlaps race on it.  Asynchronous on the handle's stream; allocates
 * nothing. */
DL_API int dl_internal_force_static(dl_handle *h, const double *u_dev,
                                    const double *theta_dev, double *fint_dev);

/* Per Gauss point history [n_elems][n_gauss]: plastic strain (6), hardening
 * parameters (up to 7), dissipated energy; any may be NULL.
 * (ElastoPlasticRodMaterial::getTable "plast_strain"/"hard_params",
 *  ElastoPlasticRodMaterial.cpp:318-364) */
DL_API int dl_get_history(dl_handle *h, double *plastic_strain,
                          double *hard_params, double *dissipation);

/* Sum of internal force (the reference's "resp": the internal force of the
 * last step, i.e. of the state before it, with contact and the gyroscopic
 * moment) and of external load per DOF over a node set
 * (GroupOutputModule.cpp:155-162): out_resp[6], out_load[6].
 * out_resp needs recording switched on (dl_set_group_output) before the
 * dl_run whose last step it reports; with recording off and out_resp
 * non-NULL the call fails with DL_ERR_INVALID.  out_load needs no recording. */

DL_API int dl_group_sums(dl_handle *h, int32_t n_nodes, const int32_t *nodes,
                         double *out_resp, double *out_load);

/* Switch recording of the last step's internal force (for dl_group_sums'
 * out_resp) on (1) or off (0).  Off by default: recording adds a store of
 * 6 doubles per node to the last step of every dl_run and selects the
 * kernel variant that carries the optional terms.  No reference counterpart
 * (GroupOutputModule reads the global internal-force vector, which the
 * reference keeps anyway). */
DL_API int dl_set_group_output(dl_handle *h, int32_t on);

/* ------------------------------------------------------------------ */
/* batching: many independent lattices in one launch                   */
/* ------------------------------------------------------------------ */

/* Create one engine holding n independent lattices, stepped together by dl_run in
 * one launch: the disjoint union of their meshes, each lattice with its own
 * deltaTime and BCs (engine feature: the reference runs one lattice per
 * process).  They must share the Gauss rule, the rotation-update options and
 * the material law.  Node numbering of the batch = concatenation of the
 * lattices' numberings (offsets from dl_batch_sizes); dl_get_state and
 * dl_set_state act on all nodes; samples record totals over all lattices. */
DL_API int dl_create_batch(const dl_model_desc *descs, int32_t n, int precision,
                           dl_handle **out);
/* n_lattices, and the node/element offsets [n_lattices + 1] of each lattice. */
DL_API int dl_batch_sizes(dl_handle *h, int32_t *n_lattices, int32_t *node_offsets,
                          int32_t *elem_offsets);
/* State of one lattice in its own node numbering (arrays sized for its nodes). */
DL_API int dl_batch_get_state(dl_handle *h, int32_t lattice, double *u,
                              double *theta, double *v);
/* Energies of one lattice at the final step of the last dl_run. */
DL_API int dl_batch_get_energies(dl_handle *h, int32_t lattice, dl_energies *e);

/* ------------------------------------------------------------------ */
/* contact                                                             */
/* ------------------------------------------------------------------ */

/* Element pairs whose contact was closed in the final step of the last
 * dl_run (element indices in the caller's numbering, a < b, sorted), with the
 * gap d - 2r.  n_pairs receives the count; at most max_pairs are written.
 * (RodContactModel::computeContacts_, RodContactModel.cpp:451-738) */
DL_API int dl_contact_pairs(dl_handle *h, int64_t *n_pairs, int32_t *pairs,
                            double *gaps, int64_t max_pairs);

/* Joint pairs in contact in the final step of the last dl_run (node indices
 * in the caller's numbering, a < b, sorted), with the gap d - 2r: the pairs
 * JointContactModel::findContacts_ finds (JointContactModel.cpp:236-275).
 * n_pairs receives the count; at most max_pairs are written. */
DL_API int dl_joint_contact_pairs(dl_handle *h, int64_t *n_pairs, int32_t *pairs,
                                  double *gaps, int64_t max_pairs);

/* Force of each rigid plate on the lattice nodes in the final step of the last
 * dl_run (internal-force sign): out[2][3].  Engine extension. */
DL_API int dl_plate_reaction(dl_handle *h, double *out);

/* Candidate-list statistics of the engine's broad phase (engine extension):
 * element pairs in the current rod-contact candidate list and list builds so
 * far (the rod and joint lists are rebuilt together). */
DL_API int dl_contact_stats(dl_handle *h, int64_t *n_candidates, int64_t *n_builds);

/* Kernels this handle has launched so far in dl_run (step kernels, the
 * external-work finisher, contact-list kernels); for benchmark reports.
 * Engine extension. */
DL_API int dl_launch_count(dl_handle *h, int64_t *n);

/* Random fibre network (engine extension; the reference reads meshes from
 * .geo/.msh files and has no generator): n_rods straight rods of the given
 * length, centres uniform in [0, box]^3, directions uniform on the sphere,
 * elems_per_rod two-node elements each; a rod closer than 2*radius to an
 * accepted rod is resampled.  Outputs: coords[n_rods*(elems_per_rod+1)][3],
 * conn[n_rods*elems_per_rod][2], elem_rod[n_rods*elems_per_rod]; tries_out
 * (optional) = rods sampled.  max_tries > 0 bounds the sampling
 * (DL_ERR_UNSUPPORTED when reached).  Same seed, same network. */
DL_API int dl_generate_fibres(int32_t n_rods, double length,
                              int32_t elems_per_rod, double radius, double box,
                              uint64_t seed, int64_t max_tries, double *coords,
                              int32_t *conn, int32_t *elem_rod,
                              int64_t *tries_out);

/* ------------------------------------------------------------------ */
/* differentiation                                                     */
/* ------------------------------------------------------------------ */

/* Forward run of nsteps from the current state storing checkpoints every
 * `checkpoint_every` steps, then the reverse sweep (each segment recomputed
 * once with a state tape): objective
 *   J = E_diss(T) + react_weight * max_k |R(k)|,
 *   R(k) = sum over react_nodes of the internal force component react_dof
 *          of step k (the group's "resp" sum, GroupOutputModule), so that
 *          max_k |R(k)| is the peak reaction force of the group,
 * and its gradient with respect to the element radii (circular sections;
 * elements sharing a parameter through elem_param[] -- e.g. the elements of
 * one strut -- have dJ/dp_k summed; elem_param may be NULL with
 * n_params = n_elems).  The handle ends in the forward run's final state.
 * checkpoint_every = 0 evaluates the objective only (grad set to zero).
 * When the state of every step fits the tape budget (dl_set_tape_budget) the
 * forward run keeps it and no segment is recomputed.  Single lattices without
 * contact.  Engine feature without counterpart in the reference. */
DL_API int dl_adjoint_radius(dl_handle *h, int64_t nsteps, int32_t checkpoint_every,
                             int32_t n_params, const int32_t *elem_param,
                             int32_t n_react_nodes, const int32_t *react_nodes,
                             int32_t react_dof, double react_weight,
                             double *objective, double *grad);

/* Branch tape of the adjoint's forward run (engine feature, no counterpart in
 * the reference).  J is piecewise smooth: a Gauss point that starts or stops
 * yielding, a change of the cutting plane's iteration count and a change of
 * the peak step all switch branches.  The adjoint differentiates the branch
 * that its forward run takes; the tape makes that branch reproducible, so
 * that finite differences can be taken along it.
 * mode 1: the next dl_adjoint_radius records the iteration count of every
 *   Gauss point in every step ([nsteps][n_gauss][n_elems] bytes, engine
 *   element order) and the peak step and sign of R;
 * mode 2: the next dl_adjoint_radius (checkpoint_every = 0: objective only)
 *   imposes the tape set by dl_adjoint_branch_tape in place of the stop test
 *   f < precision and evaluates the peak term at the imposed step as
 *   sign * R(step);
 * mode 0: off (default). */
DL_API int dl_adjoint_branch_mode(dl_handle *h, int32_t mode);
/* get != 0: copy the recorded tape (bytes = its size, see
 * dl_adjoint_branch_bytes; tape may be NULL to read the peak only) and the
 * peak step (1-based within the run) and sign; get = 0: set the tape, peak
 * step and sign to impose (e.g. recorded on another handle of the same mesh). */
DL_API int dl_adjoint_branch_tape(dl_handle *h, int32_t get, uint8_t *tape, int64_t bytes,
                                  int64_t *peak_step, double *peak_sign);
DL_API int dl_adjoint_branch_bytes(dl_handle *h, int64_t *bytes);

/* Device memory the adjoint may use for its state tape: -1 (default) half of
 * the free memory at the call, 0 checkpoints only (every segment recomputed).
 * Engine extension. */
DL_API int dl_set_tape_budget(dl_handle *h, int64_t bytes);

/* The adjoint's checkpoints and state tape come from a process-wide pool per
 * device that keeps freed memory, so a gradient evaluation on a new handle
 * (new radii) maps no fresh pages.  This call returns the pool's unused
 * memory on the current device to the driver.  No reference counterpart. */
DL_API int dl_trim_retained_memory(void);

/* ------------------------------------------------------------------ */
/* input surface helpers                                               */
/* ------------------------------------------------------------------ */

/* Source code the engine generates for a yield function (engine extension,
 * for inspection and tests): the policy of the step kernels (adjoint = 0) or
 * of the adjoint kernels with the reverse-mode product (adjoint = 1), in float
 * (fp32 = 1) or double, with device (host = 0) or inline host (host = 1)
 * member functions.  Variables are named by `names` (the argument order).
 * needed receives the length including the terminating zero. */
DL_API int dl_yield_source(const char *yield_cond, int32_t n_deriv,
                           const char *const *yield_deriv, int32_t n_vars,
                           const char *const *names, int32_t fp32,
                           int32_t adjoint, int32_t host, char *buf,
                           int64_t buf_len, int64_t *needed);

/* Evaluate an expression of the .pro language with named variables (for tests). */
DL_API int dl_eval_expression(const char *expr, int32_t n_vars,
                              const char *const *names, const double *values,
                              double *out);

/* Host-side set-up only (no device needed): element-node frames Lambda_N as
 * quaternions [n_elems][nodes_per_elem][4] (w,x,y,z), reference strains [n_elems][n_gauss][6]
 * (Gamma0, K0), node lumped mass [n_nodes] and rotational inertia at the
 * reference configuration [n_nodes][3][3] -- the quantities of
 * SpecialCosseratRodModel::initRotation_/initStrain_/assembleM_
 * (SpecialCosseratRodModel.cpp:536-658, 969-1031).  Any output may be NULL. */
DL_API int dl_inspect_setup(const dl_model_desc *desc, int precision, double *frames,
                            double *strain0, double *mass, double *rot_inertia);

/* Runtime-compile (NVRTC, no device needed) the elastoplastic step kernels and
 * the adjoint kernels of a model for sm_100a; reports the total cubin size and
 * the compiler log. */
DL_API int dl_jit_check(const dl_model_desc *desc, int precision, size_t *cubin_bytes,
                        char *log, size_t log_size);

/* Version string of the library. */
DL_API const char *dl_version(void);

/* Compute capability the library's ahead-of-time kernels were compiled for,
 * as the CUDA runtime reports it for the current device (major*10 + minor:
 * 100 for sm_100a).  Needs a device.  No counterpart in the reference. */
DL_API int dl_device_binary_version(int32_t *version);

#endif /* DYNLATTICE_H */
