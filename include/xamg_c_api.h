/*
 * XAMG C API, B200 implementation.
 *
 * Every function below has the name, argument list and meaning of the
 * reference C API (api/c/xamg_c_api.h:33-117); each declaration cites the
 * reference line it replaces. The implementation runs the solve phase on one
 * B200 GPU (sm_100a); host arrays passed in are copied, as in the reference
 * (api/c/xamg_c_api.cpp:350-373, 414-423).
 *
 * Differences a caller can observe:
 *  - Every function returns 0 on success, as in the reference; on failure it
 *    returns a negative XAMG_ERR_* code (the reference asserts instead).
 *    XAMG_b200_last_error() in xamg_b200.h gives the message.
 *  - The right-hand-side count nv is a runtime value in {1,2,4,8,16,32}
 *    (the reference fixes it at compile time with XAMG_NV);
 *    XAMG_get_nv() returns the build default XAMG_NV (1 if undefined).
 *  - There is one process and one GPU: XAMG_id_get_proc() is 0,
 *    XAMG_id_get_nprocs() is 1, XAMG_id_get_comm_ptr() returns NULL.
 */
#ifndef XAMG_C_API_H_
#define XAMG_C_API_H_

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t XAMG_param_id;          /* xamg_c_api.h:33 */
typedef size_t XAMG_param_override_id; /* xamg_c_api.h:34 */
typedef size_t XAMG_part_id;           /* xamg_c_api.h:35 */
typedef size_t XAMG_vector_id;         /* xamg_c_api.h:36 */
typedef size_t XAMG_csr_matrix_id;     /* xamg_c_api.h:37 */
typedef size_t XAMG_matrix_id;         /* xamg_c_api.h:38 */
typedef size_t XAMG_solver_id;         /* xamg_c_api.h:39 */

/* xamg_c_api.h:41 */
typedef enum { XAMG_MEM_LOCAL, XAMG_MEM_SHARED, XAMG_MEM_DISTRIBUTED } vector_alloc_mode;

int XAMG_init(int argc, char **argv, char *conf); /* xamg_c_api.h:43 */
int XAMG_finalize();                              /* xamg_c_api.h:44 */

int XAMG_get_nv(); /* xamg_c_api.h:46 */

int XAMG_id_get_proc();        /* xamg_c_api.h:48 */
int XAMG_id_get_nprocs();      /* xamg_c_api.h:49 */
void *XAMG_id_get_comm_ptr();  /* xamg_c_api.h:50 */

#define XAMG_id_get_comm() (*((MPI_Comm *)XAMG_id_get_comm_ptr())) /* xamg_c_api.h:52 */

int XAMG_param_create(XAMG_param_id *);                                               /* :54 */
int XAMG_param_add_value_s(char *solver_type, char *key, char *value, XAMG_param_id pid); /* :55 */
int XAMG_param_add_value_i(char *solver_type, char *key, uint16_t value, XAMG_param_id pid); /* :56 */
int XAMG_param_add_value_d(char *solver_type, char *key, float value, XAMG_param_id pid); /* :57 */

int XAMG_param_forced_change_value_s(char *solver_type, char *key, char *value,
                                     XAMG_param_id pid); /* :59 */
int XAMG_param_forced_change_value_i(char *solver_type, char *key, uint16_t value,
                                     XAMG_param_id pid); /* :60 */
int XAMG_param_forced_change_value_d(char *solver_type, char *key, float value,
                                     XAMG_param_id pid); /* :62 */

int XAMG_param_change_value_s(char *solver_type, char *key, char *value, XAMG_param_id pid); /* :64 */
int XAMG_param_change_value_i(char *solver_type, char *key, uint16_t value, XAMG_param_id pid); /* :65 */
int XAMG_param_change_value_d(char *solver_type, char *key, float value, XAMG_param_id pid); /* :66 */

int XAMG_param_override_create(XAMG_param_override_id *);                       /* :68 */
int XAMG_param_override_add_value(char *key, char *val, XAMG_param_override_id ovid); /* :69 */
int XAMG_param_override_apply(char *solver_type, XAMG_param_id pid,
                              XAMG_param_override_id ovid); /* :70 */
int XAMG_param_override_destroy(XAMG_param_override_id);     /* :71 */

void XAMG_param_set_default(XAMG_param_id); /* :73 */
int XAMG_param_print(XAMG_param_id);        /* :74 */
int XAMG_param_destroy(XAMG_param_id);      /* :75 */

int XAMG_part_create(XAMG_part_id *);           /* :77 */
int XAMG_part_construct(int, XAMG_part_id);     /* :78 */
int XAMG_part_get_numa_size(XAMG_part_id);      /* :79 */
int XAMG_part_destroy(XAMG_part_id);            /* :80 */

int XAMG_vector_create(XAMG_vector_id *, vector_alloc_mode);                         /* :82 */
int XAMG_vector_offset(uint64_t, XAMG_vector_id);                                     /* :83 */
int XAMG_vector_alloc_d(int, uint16_t, XAMG_vector_id);                               /* :84 */
int XAMG_vector_set_part(XAMG_part_id, XAMG_vector_id);                               /* :86 */
int XAMG_vector_set_val_d(double, XAMG_vector_id);                                    /* :87 */
int XAMG_vector_download_d(double *, uint64_t, uint64_t, uint16_t, XAMG_vector_id);   /* :88 */
int XAMG_vector_upload_v(XAMG_vector_id, XAMG_vector_id);                             /* :90 */
int XAMG_vector_upload_d(double *, uint64_t, uint64_t, uint16_t, XAMG_vector_id);     /* :91 */
int XAMG_vector_destroy(XAMG_vector_id);                                              /* :93 */

int XAMG_csr_matrix_create(XAMG_csr_matrix_id *);                  /* :95 */
int XAMG_csr_matrix_alloc(uint64_t, uint64_t, XAMG_csr_matrix_id); /* :96 */
int XAMG_csr_matrix_fill(int *, int *, double *, XAMG_matrix_id);  /* :97 */
int XAMG_csr_matrix_offset(int, int, XAMG_matrix_id);              /* :98 */
uint32_t XAMG_csr_matrix_get_nrows(XAMG_csr_matrix_id);            /* :99 */
int XAMG_csr_matrix_destroy(XAMG_csr_matrix_id);                   /* :100 */

int XAMG_matrix_create(XAMG_matrix_id *);                                  /* :102 */
int XAMG_matrix_set_part(XAMG_part_id, XAMG_matrix_id);                    /* :103 */
int XAMG_matrix_construct(XAMG_csr_matrix_id mcsrid, XAMG_matrix_id mid);  /* :104 */
int XAMG_matrix_destroy(XAMG_matrix_id);                                   /* :105 */

int XAMG_solver_create1(XAMG_matrix_id, XAMG_param_id, XAMG_solver_id *); /* :107 */
int XAMG_solver_create2(XAMG_matrix_id, XAMG_param_id, XAMG_vector_id, XAMG_vector_id,
                        XAMG_solver_id *);                                 /* :108 */
int XAMG_solver_renew_params(XAMG_param_id, XAMG_solver_id);               /* :110 */
int XAMG_solver_solve1(uint16_t, XAMG_solver_id);                          /* :111 */
int XAMG_solver_solve2(uint16_t, XAMG_vector_id, XAMG_vector_id, XAMG_solver_id); /* :112 */
int XAMG_solver_get_convergence_info(int *, uint16_t, XAMG_solver_id);    /* :113 */
int XAMG_solver_destroy(XAMG_solver_id);                                   /* :114 */

double XAMG_timer();   /* :116 */
int XAMG_barrier();    /* :117 */

#ifdef __cplusplus
}
#endif

#endif /* XAMG_C_API_H_ */
