/*
 * Implementation-defined extensions of the B200 TAPP library.
 *
 * Everything here sits in the ranges the TAPP headers leave to
 * implementations: attribute keys and error codes at or above 0x1000
 * (api/include/tapp/datatype.h:9-12 of the reference states the rule for
 * data types; this library applies it to keys and codes as well).
 * None of it is needed to use the library as a drop-in: a caller that only
 * uses the reference's API gets synchronous execution on the CUDA legacy
 * default stream with the precision the product asks for.
 */
#ifndef TAPP_B200_H_
#define TAPP_B200_H_

#include "tapp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes (returned by TAPP_execute_product and friends) ---- */
enum {
    TAPP_B200_ERR_CUDA = 0x1001,        /* a CUDA call failed (no device, launch error) */
    TAPP_B200_ERR_LIMIT = 0x1002,       /* more modes than the planner supports */
    TAPP_B200_ERR_UNSUPPORTED = 0x1003, /* storage type or option not supported */
    TAPP_B200_ERR_NOMEM = 0x1004,       /* device allocation failed */
    TAPP_B200_ERR_INVALID = 0x1005,     /* invalid object or argument */
    TAPP_B200_ERR_LABELS = 0x1006,      /* a tensor gained modes after the product was created */
    TAPP_B200_ERR_SCRATCH = 0x1007,     /* the product needs more scratch than the fixed array of
                                         * tapp_b200_execute_product_noalloc holds */
    TAPP_B200_ERR_BUDGET = 0x1008,      /* a served product needs more device memory than the
                                         * server's whole HBM budget */
};

/* ---- attribute keys, set with TAPP_attr_set on a TAPP_executor ---- */
enum {
    /* value: cudaStream_t. Work is issued on this stream instead of the
     * legacy default stream. */
    TAPP_B200_ATTR_STREAM = 0x1000,
    /* value: int* (0/1). 1: TAPP_execute_product returns without waiting for
     * the GPU; all operands must then be device pointers. */
    TAPP_B200_ATTR_ASYNC = 0x1001,
    /* value: int*. Arithmetic used for TAPP_F32F32_ACCUM_F32 products (and
     * TAPP_DEFAULT_PREC on binary32 data):
     *   0 plain binary32 on CUDA cores (default),
     *   1 split-bfloat16 on tensor cores: each operand is split into a
     *     bfloat16 high and low part, three products accumulate in binary32;
     *   2 the same with the operands always split into packed hi/lo panels
     *     first (one pass over each, then the GEMM);
     *   3 the same with the operands always read in place where their
     *     layout allows (binary32 storage; the GEMM splits them itself).
     * Mode 1 picks the faster of 2 and 3 for the product. */
    TAPP_B200_ATTR_F32_MODE = 0x1002,
    /* value: int*. Force an execution path: 0 automatic (default),
     * 1 CUDA-core element kernel, 2 CUDA-core reduction, 3 tiled CUDA-core
     * GEMM, 4 tensor cores, 5 sliced binary64 (needs TAPP_B200_ATTR_F64_MODE). */
    TAPP_B200_ATTR_PATH = 0x1004,
    /* value: int* (0/1). 1: TAPP_execute_product writes a status object to
     * *status, to be read with TAPP_attr_get and freed with
     * TAPP_destroy_status. */
    TAPP_B200_ATTR_WANT_STATUS = 0x1005,
    /* value: TAPP_b200_server (cast to void*), NULL to detach. Products
     * executed with this executor are queued on the server and the call
     * returns when the product has completed; concurrent callers (threads)
     * are batched together. Detach before destroying the server. */
    TAPP_B200_ATTR_SERVER = 0x1006,
    /* value: int*. Arithmetic of binary64 and complex-double products
     * (F64F64_ACCUM_F64, and DEFAULT on double data):
     *   0 native binary64 on CUDA cores (default),
     *   S in 2..16: sliced on the integer tensor cores. Every row of A and
     *     column of B is scaled by a power of two and cut into S signed
     *     7-bit digits; the digit products of total order < S are exact
     *     32-bit integer sums, added up in binary64. The result errs by at
     *     most about |alpha| K (S + 4) 2^(-7S) 2^(E_row + F_col) per element
     *     (K contracted terms, 2K for complex; |A[row,:]| < 2^E_row,
     *     |B[:,col]| < 2^F_col); S = 8 keeps about 56 bits of the largest
     *     element of each row. Inputs must be finite (a row or column with
     *     a non-finite value gives NaN). Environment: TAPP_B200_F64_MODE. */
    TAPP_B200_ATTR_F64_MODE = 0x1007,
    /* value: int*. Tile shape of grouped tensor-core products
     * (tapp_b200_execute_group, servers): 0 per shape class from the tuned
     * table (tapp_b200_load_tile_table), else by size (default), 1 256 x 256
     * tiles on SM pairs, 2 128 x 128 tiles. */
    TAPP_B200_ATTR_TILE = 0x1008,
};

/* ---- keys readable from a status object with TAPP_attr_get ---- */
enum {
    TAPP_B200_STATUS_PATH = 0x1100,      /* int: execution path taken (values above) */
    TAPP_B200_STATUS_KERNELS = 0x1101,   /* int: kernels launched */
    TAPP_B200_STATUS_FLOPS = 0x1102,     /* double: algorithmic flops (2|D||K|, 8|D||K| complex) */
    TAPP_B200_STATUS_DEVICE_US = 0x1103, /* double: device time of the launches, microseconds
                                          * (synchronous executions only) */
    TAPP_B200_STATUS_TC_MODE = 0x1104,   /* int: tensor-core operand mode (0 bf16, 1 f16, 2 split bf16,
                                          * 3 sliced 8-bit integer) */
    TAPP_B200_STATUS_MAIN_US = 0x1105,   /* double: device time of the dominant kernel (the tensor-core
                                          * GEMM, or the CUDA-core kernel), microseconds */
    /* double: a-priori error bound of the arithmetic the product ran in:
     * |D - D_exact| <= bound * (|alpha| sum|op_A(a) op_B(b)| + |beta| |c|)
     * + 2 u_D |D|, D_exact computed exactly from the operands as the
     * precision rounds them (16-bit operands, binary32 C under 16-bit
     * precisions) and u_D the unit roundoff of D's type. For the sliced
     * binary64 path the bound is relative to |alpha| 2^(E_row + F_col)
     * instead (see TAPP_B200_ATTR_F64_MODE). */
    TAPP_B200_STATUS_ERR_BOUND = 0x1106,
};

/*
 * Describes, in a NUL-terminated string, how the library would run the
 * product with the tensor infos' current contents: index classes after
 * repeated labels are merged, strides, compute type and path. Returns the
 * string length (like TAPP_explain_error: maxlen == 0 only measures). A
 * validation failure returns 0 and writes nothing. Host-only; touches no GPU.
 */
TAPP_EXPORT size_t tapp_b200_describe_plan(TAPP_tensor_product plan, TAPP_executor exec,
                                           size_t maxlen, char* out);

/*
 * Number of kernels this library launched since the process started (all
 * threads, all devices). For launch counting in benchmarks.
 */
TAPP_EXPORT long long tapp_b200_kernel_launches(void);

/*
 * Number of memory allocations (device memory from the library's pool or
 * cudaMalloc, page-locked host staging) this library asked CUDA for since
 * the process started (all threads, all devices). A diagnostic: it lets a
 * caller check that a code path allocated nothing.
 */
TAPP_EXPORT long long tapp_b200_device_allocations(void);

/*
 * Self-test of the bounded waits of the library's kernels (no counterpart in
 * the reference). On the current device, one kernel waits, with the waits
 * the tensor-core kernels use, on a flag that nothing raises and on an
 * mbarrier phase that nothing completes, limit_ms each. A wait that runs out
 * raises the kernel's abort word and returns, so the kernel ends and the
 * context stays usable; this is how a stalled product turns into an error
 * instead of a hang. *flag_wait_expired / *barrier_wait_expired are set to 1
 * when the wait gave up and raised the abort word, 0 otherwise.
 * Returns 0, TAPP_B200_ERR_INVALID (NULL outputs, limit_ms outside
 * (0, 10000]) or TAPP_B200_ERR_CUDA.
 */
TAPP_EXPORT TAPP_error tapp_b200_selftest_waits(double limit_ms, int* flag_wait_expired, int* barrier_wait_expired);

/*
 * TAPP_execute_product for callers that cannot allocate device memory while
 * they run a product: code running inside an allocator or memory manager,
 * or a program that has handed the whole device to its own pool. There is no
 * counterpart in the reference; it exists only in this library.
 *
 * Runs the tensor-core path (BF16BF16_ACCUM_F32, F16F16_ACCUM_F32/_F16, or
 * F32 with TAPP_B200_ATTR_F32_MODE = 1) with its packed-operand scratch in a
 * fixed 32 MiB device array of the library (held on every GPU that loads the
 * library until the process exits); the library calls no device allocator
 * (and no host allocator) on this path. A, B, C and D must be device
 * pointers (TAPP_B200_ERR_INVALID otherwise); other precisions return
 * TAPP_B200_ERR_UNSUPPORTED; products whose operand panels need more than the
 * array holds return TAPP_B200_ERR_SCRATCH without launching anything. The
 * first call on a device (and the first after a cudaDeviceReset) looks up the
 * array's device address with that device current: make it before any stream
 * capture. Every call shares the array, so calls whose work overlaps on the
 * GPU race. With an asynchronous executor the call returns before its kernels
 * run and cannot read their error word: a bounded wait that expired there is
 * reported (TAPP_B200_ERR_CUDA) by the next synchronous call of this entry
 * point on that device. Codes and validation are otherwise those of
 * TAPP_execute_product.
 */
TAPP_EXPORT TAPP_error tapp_b200_execute_product_noalloc(TAPP_tensor_product plan, TAPP_executor exec,
                                                         const void* alpha, const void* A, const void* B,
                                                         const void* beta, const void* C, void* D);

/*
 * A chain of products, such as the mode-n products that rebuild a tensor
 * from its Tucker core and factor matrices, run back to back on the
 * executor's stream without a host round trip between them (the reference
 * runs each product on its own; this entry point has no counterpart there).
 * Step i is the product plans[i] with alphas[i], betas[i], A[i], B[i],
 * C ? C[i] : NULL and D[i], as TAPP_execute_product takes them, except:
 *   - A[i] or B[i] NULL (i > 0): the D of step i - 1;
 *   - D[i] NULL (i < n - 1): an intermediate the library allocates in device
 *     memory for the step's D layout and frees after the chain.
 * D[n - 1] must be given. Each step is validated with the codes of
 * TAPP_execute_product (the first failing step's code is returned, earlier
 * steps have run); TAPP_B200_ERR_INVALID for missing pointers or an
 * executor attached to a server. Synchronous unless the executor is
 * asynchronous. The host waits once, after the last step.
 */
TAPP_EXPORT TAPP_error tapp_b200_execute_chain(int n, const TAPP_tensor_product* plans, TAPP_executor exec,
                                               const void* const* alphas, const void* const* betas,
                                               const void* const* A, const void* const* B,
                                               const void* const* C, void* const* D);

/*
 * Products of different plans in one call (the reference's batched product,
 * api/include/tapp/product.h:66-75, covers many products of one plan; this
 * entry point has no counterpart there). Product i is plans[i] with
 * alphas[i], betas[i], A[i], B[i], C ? C[i] : NULL and D[i] as
 * TAPP_execute_product takes them. Products that run on the tensor cores
 * from binary32 storage (BF16BF16_ACCUM_F32, F16F16_ACCUM_F32, or F32 in
 * split mode) without unary modes and with all operands on the device run
 * together in one persistent launch per tile shape (TAPP_B200_ATTR_TILE),
 * their operands read in place; every other product runs as
 * TAPP_execute_product runs it. All products are validated first, with the
 * codes of TAPP_execute_product; nothing runs if one fails. The products must
 * be independent (no D overlapping another product's operands). Synchronous
 * unless the executor is asynchronous; TAPP_B200_ERR_INVALID for missing
 * pointers or an executor attached to a server.
 */
TAPP_EXPORT TAPP_error tapp_b200_execute_group(int n, const TAPP_tensor_product* plans, TAPP_executor exec,
                                               const void* const* alphas, const void* const* betas,
                                               const void* const* A, const void* const* B,
                                               const void* const* C, void* const* D);

/*
 * Loads the table of tile shapes per shape class written by the tuner
 * (tapp_b200/tuner.py) for grouped tensor-core products with
 * TAPP_B200_ATTR_TILE = 0; NULL drops the table (sizes decide). The
 * environment variable TAPP_B200_TILE_TABLE names a table loaded at first
 * use. Returns 0, or TAPP_B200_ERR_INVALID when the file cannot be read.
 */
TAPP_EXPORT TAPP_error tapp_b200_load_tile_table(const char* path);

/*
 * A device-resident request loop for small products (no counterpart in the
 * reference, whose handle and executor are placeholders): a persistent
 * kernel of `blocks` blocks (1..256; every block takes a share of each
 * product's outputs) stays on the GPU and computes products as they are
 * submitted, with no kernel launch per product. Submission writes the
 * product's descriptor into a ring of `slots` entries in page-locked host
 * memory mapped into the device; the loop polls it, computes D, and marks
 * the entry done. After idle_ms without products the kernel returns (it
 * never spins without a bound); the next submission or wait launches it
 * again. Products must plan to the element path (small products) and have
 * device operands: TAPP_B200_ERR_UNSUPPORTED / TAPP_B200_ERR_INVALID
 * otherwise. Results equal TAPP_execute_product's bit for bit. Calls that
 * synchronise the whole device (cudaDeviceSynchronize) wait for the loop's
 * idle return. Destroy waits for the loop to return, then frees it.
 */
typedef intptr_t TAPP_b200_loop;

typedef struct tapp_b200_loop_counters {
    int64_t submitted, completed, launches;  /* launches: kernel starts (the first and every restart after idle) */
    int32_t running, pad;                    /* 1 while a launch is on the GPU */
    double p50_us, p99_us, mean_us, max_us;  /* submission to the wait that saw the product done */
} tapp_b200_loop_counters;

TAPP_EXPORT TAPP_error tapp_b200_loop_create(TAPP_b200_loop* loop, TAPP_executor exec, int blocks, int slots,
                                             double idle_ms);
TAPP_EXPORT TAPP_error tapp_b200_loop_submit(TAPP_b200_loop loop, TAPP_tensor_product plan, const void* alpha,
                                             const void* A, const void* B, const void* beta, const void* C, void* D,
                                             int64_t* ticket);
/* Returns once the product of `ticket` is done (30 s at most: TAPP_B200_ERR_CUDA). */
TAPP_EXPORT TAPP_error tapp_b200_loop_wait(TAPP_b200_loop loop, int64_t ticket);
TAPP_EXPORT TAPP_error tapp_b200_loop_stats(TAPP_b200_loop loop, tapp_b200_loop_counters* out);
TAPP_EXPORT TAPP_error tapp_b200_loop_reset_stats(TAPP_b200_loop loop);
TAPP_EXPORT TAPP_error tapp_b200_loop_destroy(TAPP_b200_loop loop);

/*
 * Serving: a request loop that runs products as they arrive on one GPU.
 * There is no counterpart in the reference (its handle and executor are
 * placeholders).
 *
 * tapp_b200_server_submit validates and plans a product on the calling
 * thread (returning the same codes TAPP_execute_product would) and queues
 * it; a scheduler thread admits queued products in arrival order while the
 * device memory they need fits the HBM budget and fewer than max_in_flight
 * are running, issues them over n_streams CUDA streams so that their work
 * overlaps on the GPU, and packs the small products of the CUDA-core element
 * path that it admits together into one grouped launch per compute domain.
 * Products that arrive while others run join at the next admission
 * (continuous batching); each product's memory and slot are released when its
 * own work has completed.
 *
 * Device memory charged against the budget: the staging copies of host
 * operands (as TAPP_execute_product stages them) and the scratch of the
 * product's kernels (tensor-core panels, split-contraction sums). Device-resident operands are used in place and not charged.
 * A product that needs more than the whole budget is refused at submission
 * with TAPP_B200_ERR_BUDGET. alpha and beta are read at submission; the
 * operands must stay valid, and D untouched, until the product completes. Results are those TAPP_execute_product gives for the same product:
 * each runs the same kernels with the same arguments.
 */
typedef intptr_t TAPP_b200_server;

typedef struct tapp_b200_server_counters {
    int64_t submitted;        /* products queued (refused ones excluded) */
    int64_t completed;        /* products finished, including failed ones */
    int64_t failed;           /* products whose launch failed */
    int64_t units;            /* launch units issued: grouped launches plus single products */
    int64_t grouped;          /* products that ran inside a grouped launch */
    int64_t budget_waits;     /* products that waited in the queue for budget to free up */
    int64_t peak_in_flight;   /* most products in flight at once */
    int64_t budget_bytes;     /* the budget */
    int64_t peak_reserved;    /* most bytes charged at once */
    double p50_us, p99_us, mean_us, max_us; /* latency, submission to completion */
    double span_s;            /* first submission to last completion, seconds */
    double requests_per_s;    /* completed / span_s */
    double flops;             /* algorithmic flops of the completed products */
} tapp_b200_server_counters;

/* Creates a server on the current CUDA device. exec (may be 0) supplies the
 * precision options (TAPP_B200_ATTR_F32_MODE, _PATH) of submitted products;
 * n_streams 1..16, max_in_flight >= 1. */
TAPP_EXPORT TAPP_error tapp_b200_server_create(TAPP_b200_server* server, TAPP_executor exec,
                                               int64_t hbm_budget_bytes, int n_streams, int max_in_flight);
/* Queues a product; *ticket identifies it for tapp_b200_server_wait. */
TAPP_EXPORT TAPP_error tapp_b200_server_submit(TAPP_b200_server server, TAPP_tensor_product plan,
                                               const void* alpha, const void* A, const void* B,
                                               const void* beta, const void* C, void* D, int64_t* ticket);
/* Waits for one product; returns its code (0, or the CUDA error of its launch). */
TAPP_EXPORT TAPP_error tapp_b200_server_wait(TAPP_b200_server server, int64_t ticket);
/* Waits for every product submitted so far; returns the first failure's code or 0. */
TAPP_EXPORT TAPP_error tapp_b200_server_drain(TAPP_b200_server server);
/* Counters and latency percentiles of the products completed so far. */
TAPP_EXPORT TAPP_error tapp_b200_server_stats(TAPP_b200_server server, tapp_b200_server_counters* out);
/* Forgets completed products (their tickets become invalid) and restarts the
 * counters; products in flight are kept. */
TAPP_EXPORT TAPP_error tapp_b200_server_reset_stats(TAPP_b200_server server);
/* Drains, stops the scheduler and frees the server. */
TAPP_EXPORT TAPP_error tapp_b200_server_destroy(TAPP_b200_server server);

#ifdef __cplusplus
}
#endif

#endif /* TAPP_B200_H_ */
