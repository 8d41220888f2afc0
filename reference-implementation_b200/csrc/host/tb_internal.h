/*
 * Internal objects of the B200 TAPP library (host side, C11).
 */
#ifndef TB_INTERNAL_H_
#define TB_INTERNAL_H_

#include <pthread.h>
#include <stdint.h>

#include "tapp.h"
#include "tapp_b200.h"
#include "../tb_plan.h"
#include "../tb_cuda.h"

#define TB_MAGIC_INFO 0x54420001
#define TB_MAGIC_PRODUCT 0x54420002
#define TB_MAGIC_HANDLE 0x54420003
#define TB_MAGIC_STATUS 0x54420005

/* tensor info: ref_impl.h:13-19 of the reference holds the same fields */
struct tb_info {
    int magic;
    TAPP_datatype type;
    int nmode;
    int64_t* extents;
    int64_t* strides;
};

/* executor: the first int is the executor id the reference's product checks
 * (1 = the reference's own executor, product.c:878-885) */
struct tb_executor {
    int id;
    int reserved;
    void* stream;          /* cudaStream_t, NULL = legacy default stream */
    int async;
    int f32_mode;
    int force_path;
    int want_status;
    struct tb_server* server;   /* TAPP_B200_ATTR_SERVER */
    int f64_mode;               /* TAPP_B200_ATTR_F64_MODE */
    int tile;                   /* TAPP_B200_ATTR_TILE */
};

struct tb_handle {
    int magic;
    int device;
};

struct tb_status {
    int magic;
    int path;
    int kernels;
    int tc_mode;
    double flops;
    double device_us;
    double main_us;
    double err_bound;
};

/* cached launch plan of a product, keyed on the infos' contents */
struct tb_plan_cache {
    int valid;
    int key_len;
    int64_t* key;
    int f32_mode, force_path, f64_mode;
    tb_plan plan;
};

/* product: ref_impl.h:21-37 of the reference; infos are kept by reference */
struct tb_product {
    int magic;
    TAPP_handle handle;
    TAPP_element_op op[4];
    TAPP_tensor_info info[4];
    int64_t* idx[4];
    int nidx[4];
    TAPP_prectype prec;
    pthread_mutex_t lock;
    struct tb_plan_cache cache;
};

/* registry of executors created by this library */
int tb_executor_is_ours(TAPP_executor e);
int tb_handle_is_ours(TAPP_handle h);

/* snapshot of one tensor at execute time */
typedef struct tb_tensor_view {
    TAPP_datatype type;
    int nmode;
    int op;
    const int64_t* extents;
    const int64_t* strides;
    const int64_t* idx;
} tb_tensor_view;

/* validate.c: the reference's check chain (product.c:199-206) without the
 * executor check; returns the first failing code or 0 */
int tb_validate(const tb_tensor_view* A, const tb_tensor_view* B,
                const tb_tensor_view* C, const tb_tensor_view* D,
                const void* beta, int C_present);
int tb_scalar_is_zero(const void* s, TAPP_datatype t);

/* planner.c */
typedef struct tb_plan_options {
    int f32_mode;     /* TAPP_B200_ATTR_F32_MODE */
    int force_path;   /* TAPP_B200_ATTR_PATH */
    int f64_mode;     /* TAPP_B200_ATTR_F64_MODE: 0 native, S >= 2 sliced */
} tb_plan_options;

int tb_build_plan(const tb_tensor_view* A, const tb_tensor_view* B,
                  const tb_tensor_view* C, const tb_tensor_view* D,
                  TAPP_prectype prec, const void* alpha, const void* beta,
                  const tb_plan_options* opt, tb_plan* out);
int tb_plan_set_scalars(tb_plan* P, const void* alpha, const void* beta);
size_t tb_describe(const tb_plan* p, size_t maxlen, char* out);
double tb_plan_flops(const tb_plan* p);
double tb_plan_error_bound(const tb_plan* p);
int tb_elem_bytes(TAPP_datatype t);
int tb_is_complex(TAPP_datatype t);

/* product.c: settings an execution runs with, and the steps of an
 * execution that the server shares */
typedef struct tb_exec_settings {
    void* stream;
    int async, f32_mode, force_path, want_status;
    struct tb_server* server;
    int f64_mode;
    int tile;     /* grouped tensor-core tile shape: 0 table / rule, 1 256x256, 2 128x128 */
} tb_exec_settings;

/* tiles.c: tile shape of a grouped tensor-core product (1: 256 x 256 on CTA
 * pairs, 2: 128 x 128) from the tuned table, else from the size rule */
int tb_tile_choice(const tb_plan* P);

int tb_product_views(struct tb_product* p, tb_tensor_view v[4]);
int tb_product_plan(struct tb_product* p, const tb_tensor_view v[4], const void* alpha, const void* beta,
                    const tb_exec_settings* s, tb_plan* out);
/* lowest and highest element offset a layout addresses (0 if none), and
 * whether every element in between is addressed */
int tb_span_of(const tb_tensor_view* t, int64_t* lo, int64_t* hi);
int tb_span_dense(const tb_tensor_view* t, int64_t lo, int64_t hi);

/* server.c */
struct tb_server;
int tb_server_is_live(const struct tb_server* srv);
int tb_server_enqueue(struct tb_server* srv, struct tb_product* p, const tb_tensor_view v[4],
                      const tb_exec_settings* s, const void* alpha, const void* A, const void* B,
                      const void* beta, const void* C, void* D, int64_t* ticket);

#endif /* TB_INTERNAL_H_ */
