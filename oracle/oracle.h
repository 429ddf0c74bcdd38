/*
 * oracle.h -- C ABI of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is an FP64 CPU restatement of
 * dynLattice's explicit path (SpecialCosseratRodModel, Line3D, helpers,
 * ElasticRod/ElastoPlasticRod materials, ExplicitModule + LeapFrogModule as
 * intended and MilneDeviceModule with ExplicitModule's step control,
 * RodContactModel force path).  Only the tests, the smoke check and
 * the CPU-baseline leg of bench.py load it; the engine never does.
 *
 * Parity status: the reference binary cannot be built here (JEM/JIVE 3.0,
 * gmsh 4.9.5, HDF5 are absent), and the reference ships no tight-tolerance
 * golden vectors -- its own tests compare against digitised literature curves
 * at 5 %.  The oracle is pinned by (a) analytic known answers (Rodrigues
 * exp/log round trips, dexp vs finite differences, rigid-motion invariance,
 * closed-form cantilever statics, fint = dE/du) and (b) the reference's
 * literature-curve tests: the transient benchmarks (explicit runs) and the
 * quasi-static plastic and contact benchmarks (through a static Newton
 * driver on orc_static_force / orc_static_commit, which pins the return map
 * and the contact force); parity of the oracle against the reference binary
 * itself is unpinned.
 */
#ifndef DL_ORACLE_H
#define DL_ORACLE_H

#include "../include/dynlattice.h"

#ifdef __cplusplus
#define ORC_API extern "C" __attribute__((visibility("default")))
#else
#define ORC_API extern __attribute__((visibility("default")))
#endif

typedef struct orc_handle_s orc_handle;

ORC_API const char *orc_last_error(void);
ORC_API int orc_set_threads(int n);
ORC_API int orc_create(const dl_model_desc *desc, orc_handle **out);
ORC_API int orc_destroy(orc_handle *h);
ORC_API int orc_run(orc_handle *h, int64_t nsteps);
ORC_API int orc_set_sampling(orc_handle *h, int32_t every, int32_t n_watch,
                             const int32_t *watch_nodes);
ORC_API int orc_get_samples(orc_handle *h, int64_t *n_samples, int64_t *steps,
                            double *node_rows, dl_energies *energies,
                            int64_t max_samples);
ORC_API int orc_get_state(orc_handle *h, double *u, double *theta, double *v);
ORC_API int orc_set_state(orc_handle *h, const double *u, const double *theta,
                          const double *v);
ORC_API int orc_get_energies(orc_handle *h, dl_energies *e);
ORC_API int orc_internal_force(orc_handle *h, const double *u,
                               const double *theta, double *fint);
ORC_API int orc_static_force(orc_handle *h, const double *u,
                             const double *theta, double *fint);
ORC_API int orc_static_commit(orc_handle *h, const double *u,
                              const double *theta);
ORC_API int orc_elastic_energy(orc_handle *h, const double *u,
                               const double *theta, double *energy);
ORC_API int orc_get_history(orc_handle *h, double *plastic_strain,
                            double *hard_params, double *dissipation);
ORC_API int orc_get_frames(orc_handle *h, double *lambda_n, double *strain0);
ORC_API int orc_mass(orc_handle *h, const double *theta, double *m_trans,
                     double *m_rot);
ORC_API int orc_error_word(orc_handle *h, uint32_t *word);
ORC_API int orc_contact_pairs(orc_handle *h, int64_t *n_pairs, int32_t *pairs,
                              double *gaps, int64_t max_pairs);
ORC_API int orc_joint_contact_pairs(orc_handle *h, int64_t *n_pairs, int32_t *pairs,
                                    double *gaps, int64_t max_pairs);
ORC_API int orc_element_table(orc_handle *h, const char *name, double *out);
ORC_API int orc_blacklist_size(orc_handle *h, int64_t *n);
ORC_API int orc_plate_reaction(orc_handle *h, double *out);
ORC_API int orc_group_sums(orc_handle *h, int32_t n_nodes, const int32_t *nodes,
                           double *out_resp, double *out_load);
ORC_API int orc_set_integrator(orc_handle *h, const dl_integrator_desc *d);
ORC_API int orc_get_time(orc_handle *h, double *t, double *dt, int64_t *step,
                         int64_t *rejected);
ORC_API int orc_get_sample_times(orc_handle *h, double *times, int64_t max_samples);

#endif
