/*
 * qcm_b200.h -- C-ABI of the B200-native two-site DMRG effective-Hamiltonian path.
 *
 * Plain C: opaque handles, host pointers and sizes, int status codes.  No
 * entry point exits the process; on failure it returns a negative code and
 * qcm_last_error() describes the cause (thread-local).
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the QCMaquis tree's dmrg/ directory).
 */
#ifndef QCM_B200_H
#define QCM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define QCM_OK 0
#define QCM_ERR_ARG (-1)      /* invalid argument (std::runtime_error in the reference) */
#define QCM_ERR_CUDA (-2)     /* CUDA runtime / launch failure (reference: exit(EXIT_FAILURE)) */
#define QCM_ERR_NOMEM (-3)    /* host or device allocation failed */
#define QCM_ERR_INTERNAL (-4) /* internal consistency error */
#define QCM_ERR_NODEV (-5)    /* no CUDA device: there is no CPU fallback */

/* Human-readable description of the last failure on this thread. */
const char* qcm_last_error(void);

/* Library version string. */
const char* qcm_version(void);

/* ------------------------------------------------------------------------ */
/* MPO (input preparation)                                                    */
/* ------------------------------------------------------------------------ */

typedef struct qcm_mpo qcm_mpo;

/* Exact TwoU1 QC Hamiltonian MPO from integrals h[L*L] and V[L^4] (chemist
 * notation (pq|rs), row-major), terms with |coefficient| <= cutoff dropped.
 * Replaces qc_model::create_terms + make_mpo
 * (framework/dmrg/models/chem/2u1/model.hpp:184, models/generate_mpo.hpp:37). */
int qcm_mpo_build_qc(int L, const double* h, const double* V, double cutoff, qcm_mpo** out);

/* Two-site MPO W_ts[p] = W[p] (x) W[p+1] contracted over the shared bond.
 * Replaces make_ts_cache_mpo / make_twosite_mpo
 * (framework/dmrg/mp_tensors/ts_ops.hpp:97-185). */
int qcm_mpo_make_twosite(const qcm_mpo* m, qcm_mpo** out);

/* Number of site tensors (L, or L-1 for a two-site MPO); -1 for NULL. */
int qcm_mpo_length(const qcm_mpo* m);

/* Binary interchange blob ("QMPO" v1).  Call with buf == NULL to get *len. */
int qcm_mpo_serialize(const qcm_mpo* m, void* buf, size_t cap, size_t* len);
int qcm_mpo_deserialize(const void* buf, size_t len, qcm_mpo** out);
void qcm_mpo_free(qcm_mpo* m);

#ifdef __cplusplus
}
#endif

#endif /* QCM_B200_H */
