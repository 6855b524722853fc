/* XAMG C API, served by the B200 solve-phase library libxamg_b200.so.
 *
 * Every declaration below has the signature of the reference's C API
 * (api/c/xamg_c_api.h:43-122 in MatveevAlexy/xamg-test), so a caller of the
 * reference relinks against this library unchanged.  Differences in behaviour:
 *   - vectors created XAMG_MEM_SHARED or XAMG_MEM_DISTRIBUTED live in GPU
 *     memory; XAMG_MEM_LOCAL vectors live in host memory, and
 *     XAMG_vector_upload_v(local, distributed) is the host-to-device copy;
 *   - the right-hand-side width NV is a runtime setting (environment variable
 *     XAMG_NV at XAMG_init, or XAMG_b200_set_nv) instead of the compile-time
 *     XAMG_NV macro; functions taking nv check it against that setting;
 *   - errors return a non-zero code (2 bad argument, 3 CUDA error, 4 method not
 *     available on the device path) instead of asserting; the message is kept
 *     for XAMG_b200_last_error();
 *   - there is one process per GPU: XAMG_id_get_nprocs() is 1 and
 *     XAMG_id_get_comm_ptr() returns NULL.
 */
#ifndef XAMG_C_API_H_
#define XAMG_C_API_H_

#include <stdint.h>
#include <stdlib.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t XAMG_param_id;
typedef size_t XAMG_param_override_id;
typedef size_t XAMG_part_id;
typedef size_t XAMG_vector_id;
typedef size_t XAMG_csr_matrix_id;
typedef size_t XAMG_matrix_id;
typedef size_t XAMG_solver_id;

typedef enum { XAMG_MEM_LOCAL, XAMG_MEM_SHARED, XAMG_MEM_DISTRIBUTED } vector_alloc_mode;

/* api/c/xamg_c_api.h:43-50 */
int XAMG_init(int argc, char **argv, char *conf);
int XAMG_finalize();
int XAMG_get_nv();
int XAMG_id_get_proc();
int XAMG_id_get_nprocs();
void *XAMG_id_get_comm_ptr();

/* api/c/xamg_c_api.h:54-79: parameter lists */
int XAMG_param_create(XAMG_param_id *);
int XAMG_param_add_value_s(char *solver_type, char *key, char *value, XAMG_param_id pid);
int XAMG_param_add_value_i(char *solver_type, char *key, uint32_t value, XAMG_param_id pid);
int XAMG_param_add_value_d(char *solver_type, char *key, double value, XAMG_param_id pid);
int XAMG_param_add_value_b(char *solver_type, char *key, uint8_t value, XAMG_param_id pid);
int XAMG_param_forced_change_value_s(char *solver_type, char *key, char *value, XAMG_param_id pid);
int XAMG_param_forced_change_value_i(char *solver_type, char *key, uint32_t value,
                                     XAMG_param_id pid);
int XAMG_param_forced_change_value_d(char *solver_type, char *key, double value, XAMG_param_id pid);
int XAMG_param_forced_change_value_b(char *solver_type, char *key, uint8_t value,
                                     XAMG_param_id pid);
int XAMG_param_change_value_s(char *solver_type, char *key, char *value, XAMG_param_id pid);
int XAMG_param_change_value_i(char *solver_type, char *key, uint32_t value, XAMG_param_id pid);
int XAMG_param_change_value_d(char *solver_type, char *key, double value, XAMG_param_id pid);
int XAMG_param_change_value_b(char *solver_type, char *key, uint8_t value, XAMG_param_id pid);
int XAMG_param_override_create(XAMG_param_override_id *);
int XAMG_param_override_add_value(char *key, char *val, XAMG_param_override_id ovid);
int XAMG_param_override_apply(char *solver_type, XAMG_param_id pid, XAMG_param_override_id ovid);
int XAMG_param_override_destroy(XAMG_param_override_id);
void XAMG_param_set_default(XAMG_param_id);
int XAMG_param_print(XAMG_param_id);
int XAMG_param_destroy(XAMG_param_id);

/* api/c/xamg_c_api.h:81-84: partitioner (one block per process) */
int XAMG_part_create(XAMG_part_id *);
int XAMG_part_construct(int, XAMG_part_id);
int XAMG_part_get_numa_size(XAMG_part_id);
int XAMG_part_destroy(XAMG_part_id);

/* api/c/xamg_c_api.h:86-97: block vectors (size x nv, row-major) */
int XAMG_vector_create(XAMG_vector_id *, vector_alloc_mode);
int XAMG_vector_offset(uint64_t, XAMG_vector_id);
int XAMG_vector_alloc_d(int, uint16_t, XAMG_vector_id);
int XAMG_vector_set_part(XAMG_part_id, XAMG_vector_id);
int XAMG_vector_set_val_d(double, XAMG_vector_id);
int XAMG_vector_download_d(double *, uint64_t, uint64_t, uint16_t, XAMG_vector_id);
int XAMG_vector_upload_v(XAMG_vector_id, XAMG_vector_id);
int XAMG_vector_upload_d(double *, uint64_t, uint64_t, uint16_t, XAMG_vector_id);
int XAMG_vector_destroy(XAMG_vector_id);

/* api/c/xamg_c_api.h:99-104: host CSR matrices */
int XAMG_csr_matrix_create(XAMG_csr_matrix_id *);
int XAMG_csr_matrix_alloc(uint64_t, uint64_t, uint64_t, XAMG_csr_matrix_id);
int XAMG_csr_matrix_fill(int *, int *, double *, XAMG_matrix_id);
int XAMG_csr_matrix_offset(int, int, XAMG_matrix_id);
uint32_t XAMG_csr_matrix_get_nrows(XAMG_csr_matrix_id);
int XAMG_csr_matrix_destroy(XAMG_csr_matrix_id);

/* api/c/xamg_c_api.h:106-109: device matrices */
int XAMG_matrix_create(XAMG_matrix_id *);
int XAMG_matrix_set_part(XAMG_part_id, XAMG_matrix_id);
int XAMG_matrix_construct(XAMG_csr_matrix_id mcsrid, XAMG_matrix_id mid);
int XAMG_matrix_destroy(XAMG_matrix_id);

/* api/c/xamg_c_api.h:111-120: solvers */
int XAMG_solver_create1(XAMG_matrix_id, XAMG_param_id, XAMG_solver_id *);
int XAMG_solver_create2(XAMG_matrix_id, XAMG_param_id, XAMG_vector_id, XAMG_vector_id,
                        XAMG_solver_id *);
int XAMG_solver_renew_params(XAMG_param_id, XAMG_solver_id);
int XAMG_solver_solve1(uint16_t, XAMG_solver_id);
int XAMG_solver_solve2(uint16_t, XAMG_vector_id, XAMG_vector_id, XAMG_solver_id);
int XAMG_solver_print_info(XAMG_solver_id);
int XAMG_solver_get_convergence_info(int *, uint16_t, XAMG_solver_id);
int XAMG_solver_get_iter_info(int *, XAMG_solver_id);
int XAMG_solver_destroy(XAMG_solver_id);

/* api/c/xamg_c_api.h:122-123 */
double XAMG_timer();
int XAMG_barrier();

#ifdef __cplusplus
}
#endif

#endif /* XAMG_C_API_H_ */
