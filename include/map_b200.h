/*
 * map_b200.h -- C ABI of the B200 map-algebra engine (libmap_b200.so).
 *
 * The first block of functions is the reference's C ABI, same names, argument
 * order and by-value POD structs, so that its ctypes bindings (python/map.py)
 * and C/C++ callers bind unchanged. Each declaration cites the reference
 * declaration it replaces (front/bindings.hpp:<line>).
 *
 * Error behaviour: the reference asserts; this library never aborts on bad input.
 * A function that fails returns NULL (node constructors), a non-zero int
 * (ma_write) or an empty value, and records a message readable through
 * ma_lastError(); ma_errorCode() is non-zero after a failure and is cleared by
 * the next successful call.
 */
#ifndef MAP_B200_H_
#define MAP_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Scalar value + data type tag, 16 bytes, by value (util/VariantType.hpp:20-40). */
typedef struct ma_Variant {
  union {
    float f32; double f64; uint8_t b8; uint8_t u8; uint16_t u16; uint32_t u32; uint64_t u64;
    int8_t s8; int16_t s16; int32_t s32; int64_t s64;
  } u;
  int dtype;
} ma_Variant;

/* Two ints + count, 12 bytes, by value (util/Array4.hpp:42-45): data sizes,
 * block sizes and coordinates. An empty array (n == 0) denotes D0. */
typedef struct ma_Array {
  int arr[2];
  int n;
} ma_Array;

typedef struct ma_Node ma_Node; /* opaque IR node owned by the runtime */

/* ---- reference ABI ---------------------------------------------------- */

void ma_setupDevices(const char *plat_name, int dev_type, const char *dev_name); /* front/bindings.hpp:27 */
void ma_increaseRef(ma_Node *node);                                              /* front/bindings.hpp:29 */
void ma_decreaseRef(ma_Node *node);                                              /* front/bindings.hpp:30 */
void ma_eval(ma_Node **vec, int num);                                            /* front/bindings.hpp:32 */
ma_Variant ma_value(ma_Node *node);                                              /* front/bindings.hpp:33 */
int ma_nodeid(ma_Node *node);                                                    /* front/bindings.hpp:36 */
int ma_datatype(ma_Node *node);                                                  /* front/bindings.hpp:38 */
int ma_numdim(ma_Node *node);                                                    /* front/bindings.hpp:39 */
int ma_memorder(ma_Node *node);                                                  /* front/bindings.hpp:40 */
ma_Array ma_datasize(ma_Node *node);                                             /* front/bindings.hpp:41 */
ma_Array ma_blocksize(ma_Node *node);                                            /* front/bindings.hpp:42 */
ma_Node *ma_read(const char *file_path);                                         /* front/bindings.hpp:48 */
int ma_write(ma_Node *node, const char *file_path);                              /* front/bindings.hpp:49 */
ma_Node *ma_constant(ma_Variant var, ma_Array ds, int dt, int mo, ma_Array bs);  /* front/bindings.hpp:55 */
ma_Node *ma_rand(ma_Node *seed, int dt, int mo);                                 /* front/bindings.hpp:56 */
ma_Node *ma_cast(ma_Node *node, int type);                                       /* front/bindings.hpp:57 */
ma_Node *ma_index(ma_Node *node, int dim);                                       /* front/bindings.hpp:58 */
ma_Node *ma_conditional(ma_Node *cond, ma_Node *lhs, ma_Node *rhs);              /* front/bindings.hpp:59 */
ma_Node *ma_unary(ma_Node *node, int type);                                      /* front/bindings.hpp:61 */
ma_Node *ma_binary(ma_Node *lhs, ma_Node *rhs, int type);                        /* front/bindings.hpp:62 */
ma_Node *ma_diversity(ma_Node **vec, int num, int type);                         /* front/bindings.hpp:63 */
ma_Node *ma_access(ma_Node *node, ma_Array coord);                               /* front/bindings.hpp:65 */
ma_Node *ma_lhsAccess(ma_Node *lhs, ma_Node *rhs, ma_Array coord);               /* front/bindings.hpp:66 */
ma_Node *ma_neighbor(ma_Node *node, ma_Array coord);                             /* front/bindings.hpp:68 */
ma_Node *ma_boundedNbh(ma_Node *node, ma_Node *cx, ma_Node *cy);                 /* front/bindings.hpp:69 */
ma_Node *ma_spreadNeighbor(ma_Node *node, ma_Node *dir, int type);               /* front/bindings.hpp:70 */
ma_Node *ma_convolution(ma_Node *node, ma_Variant *mask_v, int mask_s, ma_Array mask_ds);           /* :71 */
ma_Node *ma_focalFunc(ma_Node *node, ma_Variant *mask_v, int mask_s, ma_Array mask_ds, int type);   /* :72 */
ma_Node *ma_focalPercent(ma_Node *node, ma_Variant *mask_v, int mask_s, ma_Array mask_ds, int type); /* :73 */
ma_Node *ma_zonalReduc(ma_Node *node, int type);                                 /* front/bindings.hpp:75 */
ma_Node *ma_radialScan(ma_Node *node, int type, ma_Array coord);                 /* front/bindings.hpp:76 */
ma_Node *ma_spreadScan(ma_Node *node, ma_Node *dir, int type);                   /* front/bindings.hpp:77 */
ma_Node *ma_stats(ma_Node *node);                                                /* front/bindings.hpp:79 */
ma_Node *ma_barrier(ma_Node *node);                                              /* front/bindings.hpp:80 */
/* Symbolic loops: the reference captures a Python `while` over a raster
 * condition through these entries (python/map.py:234-330, assembled by
 * runtime/Runtime.cpp:156-311) but has no task to run the loop
 * (runtime/task/Task.cpp:38-84). Here the Python module runs such loops itself,
 * one evaluation per iteration with the loop-carried rasters kept resident by
 * ma_materialize; these capture entries record an "unsupported" error. */
void ma_loopStart(void);                                                         /* front/bindings.hpp:86 */
void ma_loopCond(ma_Node *cond);                                                 /* front/bindings.hpp:87 */
void ma_loopBody(void);                                                          /* front/bindings.hpp:88 */
void ma_loopAgain(void);                                                         /* front/bindings.hpp:89 */
ma_Node *ma_loopAssemble(void);                                                  /* front/bindings.hpp:90 */
void ma_loopEnd(void);                                                           /* front/bindings.hpp:91 */
void ma_loopAgainTail(ma_Node *loop, ma_Node ***agains, ma_Node ***tails, int *num); /* front/bindings.hpp:92 */

/* Called by python/map.py (Raster.streamdir / Raster.numblock) but absent from
 * the reference library; provided so those methods work. */
int ma_streamdir(ma_Node *node);
ma_Array ma_numblock(ma_Node *node);

/* ---- extensions (no counterpart in the reference) ------------------------ */

const char *ma_lastError(void);   /* message of the last failure on this thread */
int ma_errorCode(void);           /* 0 after a successful call, non-zero after a failure */
void ma_clearError(void);

/* Border rule of focal reads outside the raster: 0 block mirror (reference),
 * 1 raster-edge mirror, 2 dead (zero). Applies to evaluations that follow. */
void ma_setBorder(int mode);
int ma_getBorder(void);
/* Launch granularity: 0 one launch per group over the whole raster (default),
 * 1 one launch per group per block in the scheduler's order (reference granularity). */
void ma_setExecMode(int mode);
int ma_getExecMode(void);
/* Streamed evaluation: a program whose outputs go to host memory and whose
 * groups are Local / Focal runs in row bands, each band's upload, kernels and
 * download on their own streams so the host<->device copies of successive
 * bands overlap each other and the kernels; rasters larger than device memory
 * work this way too. rows = 0 chooses bands automatically (about 32 MiB of
 * host traffic per band, used when a raster has at least four bands), rows > 0
 * forces bands of that many rows, rows < 0 turns streaming off. Results are
 * identical to whole-raster evaluation. */
void ma_setStreamRows(int rows);
int ma_getStreamRows(void);
/* Packed cells: focal groups with float math compute the cells of two rows per
 * thread step, their float additions, subtractions, multiplications and the
 * polynomial parts of sin, cos and atan2 as packed f32x2 instructions; focal
 * groups of integer arithmetic on byte rasters whose values provably stay in
 * [0, 0x7FFF] (Life, thresholds of small-weight correlations) compute four
 * cells of a row per step as 16-bit lanes of two words. Results are
 * bit-identical either way; on = 0 computes one cell at a time. Engine option
 * with no counterpart in the reference. */
void ma_setPairedCells(int on);
int ma_getPairedCells(void);
/* Flow accumulations (spreadScan) of integer water over more than 64 K cells
 * and at most `cells` cells run as pointer jumping over the Euler tour of the
 * D8 forest: about log2(2N) rounds whatever the length of the longest flow
 * path, O(N log N) work. Other rasters walk the flow paths (O(N) work, one
 * atomic step per cell of the longest path), which is faster for a whole
 * raster on an idle GPU; serving windows above 64 K cells always jump (they
 * run beside other requests, where the fixed rounds cut the latency tail).
 * Results are identical (integer sums). cells < 0 restores the default (0, or
 * MAP_B200_SPREAD_PJ), 0 never jumps. A direction raster with a cycle makes the
 * jumping form fail with an error. Engine option with no counterpart in the
 * reference. */
void ma_setFlowJumpCells(long long cells);
long long ma_getFlowJumpCells(void);
/* Algebraic rewrite of hillshade compositions (python/hill.py:41-49):
 * cz cos(atan(k sqrt(x^2+y^2))) + sz sin(...) cos(ar - aspect(x, y)) is
 * generated as (cz + sz k (y S - x C)) / sqrt(1 + k^2 (x^2 + y^2)), with the
 * script's wrap constants (its PI = 3.141593) folded into S and C, so the
 * kernel evaluates no transcendental function per cell. Results stay within
 * the hillshade tolerance of the literal chain; cells where x^2 + y^2 is not
 * finite take the literal chain. When the derivatives are correlations of
 * one input with weights 0 or +-2^k scaled by a power of two (hill.py's
 * Sobel / 8), they are also computed without their zero-weight terms and
 * folded into the constants (bit-identical on finite cells; on = 2 turns this
 * part off). on = 0 generates the literal chain everywhere. Engine option
 * with no counterpart in the reference. */
/* Prediction (runtime/visitor/Predictor.cpp:22-200, runtime/Worker.cpp:83-91):
 * a Local / Focal group whose every output holds one value known on the host
 * (constants, element-wise operators of them, focal operators of them under a
 * mirror border rule) is written with a fill instead of a kernel launch. On by
 * default; ma_lastPredictedCount() counts the groups of the last evaluation
 * that were filled. */
void ma_setPrediction(int on);
int ma_getPrediction(void);
int ma_lastPredictedCount(void);
void ma_setAlgebraicRewrite(int on);
int ma_getAlgebraicRewrite(void);
/* Block size given to rasters created without one (default 256 x 256). */
void ma_setDefaultBlockSize(ma_Array bs);
void ma_setDevice(int device);

/* D8 steepest-descent flow direction (U8 codes 1 << dir, dir in E, SE, S, SW,
 * W, NW, N, NE order; 0 for pits and flats). The reference builds the node in
 * C++ only (front/Raster.cpp:485-557, FocalFlow::Factory) with no C binding. */
ma_Node *ma_focalFlow(ma_Node *node);

/* Radial scan limited to fronts within `radius` cells of the start along the
 * octant's primary axis (radius <= 0: the whole raster). Cells not swept hold
 * NaN (all-ones bytes) in every output of the scan's group. */
ma_Node *ma_radialScanRadius(ma_Node *node, int type, ma_Array coord, double radius);

/* Raster inputs from caller memory. `data` is dense row-major (ds.arr[0]
 * columns, ds.arr[1] rows). ma_fromHost copies the cells when copy != 0,
 * otherwise it keeps the pointer, which must stay valid while the node is used
 * (pinned memory from ma_hostAlloc makes the upload asynchronous). */
ma_Node *ma_fromHost(const void *data, ma_Array ds, int dt, ma_Array bs, int copy);
/* Device-resident raster input (pitch in bytes); the memory is not copied.
 * The library works on its own CUDA stream (ma_stream), which does not wait for
 * other streams: work that writes the memory (or an output buffer it is given)
 * must be complete, or ordered before ma_stream() by an event, when the
 * evaluation is enqueued. */
ma_Node *ma_fromDevice(void *dptr, long long pitch, ma_Array ds, int dt, ma_Array bs);

/* Row bands (splitting one raster over several devices or processes; no
 * counterpart in the reference, whose runtime forces one device,
 * runtime/Runtime.cpp:110-111).
 * ma_fromDeviceRows: a device input holding only rows [row0, row0 + rows) of a
 *   ds raster, `dptr` the address of row row0 (16-byte aligned, pitch a
 *   multiple of 16 bytes). Such an input is evaluated by ma_evalRows only.
 * ma_evalRows: evaluates rows [y0, y1) of the n rasters into device memory
 *   dst[i] (the address of row y0, pitch[i] bytes between rows). The program
 *   must consist of Local and Focal groups over one raster shape, with device
 *   inputs holding at least rows [y0 - m, y1 + m) (clipped to the raster),
 *   m = ma_rowMargin(...). Border rules are applied in whole-raster
 *   coordinates, so the rows equal those of a whole-raster evaluation.
 *   Returns 0 on success and blocks until the rows are written.
 * ma_rowMargin: m for the program computing the n rasters (no device needed),
 *   or -1 with the reason in ma_lastError(). */
ma_Node *ma_fromDeviceRows(void *dptr, long long pitch, ma_Array ds, int dt, ma_Array bs, int row0, int rows);
int ma_evalRows(ma_Node **nodes, int n, void **dst, const long long *pitch, int y0, int y1);
int ma_rowMargin(ma_Node **nodes, int n);

/* `.bin` raster files (file/binary.cpp:221-404) on the host, no device needed:
 * ma_binInfo fills info7 with data type, number of dimensions, data size
 * (x, y), memory order and block size (x, y) from the header; ma_binReadHost
 * reads the cells as a dense row-major array; ma_binWriteHost writes one
 * (memory order ROW + BLK: block by block, edge blocks padded; ROW: dense).
 * Engine extension: the reference reads and writes these files only inside
 * evaluations (Read / Write nodes). Return 0 on success. */
int ma_binInfo(const char *path, int *info7);
int ma_binReadHost(const char *path, void *dst, size_t bytes);
int ma_binWriteHost(const char *path, const void *src, ma_Array ds, int dt, int mo, ma_Array bs);

/* Evaluate `node` and copy the raster to dense row-major host memory of
 * `bytes` bytes. Returns 0 on success. */
int ma_toHost(ma_Node *node, void *dst, size_t bytes);
/* Evaluate `node` into device memory (written in place when possible).
 * With async != 0 the call returns once the work is enqueued on the library's
 * stream (see ma_stream / ma_sync). Returns 0 on success. */
int ma_toDevice(ma_Node *node, void *dptr, long long pitch, int async);
/* Evaluate the `num` nodes of `vec` in one evaluation and write to out[i] a
 * node that holds the value of vec[i]: a 2-D raster kept in a device buffer
 * the library owns (freed, stream-ordered, once the node is unreferenced and
 * ma_collectGarbage runs), a scalar (D0) as a constant. Device inputs holding a
 * whole raster and constants come back as they are. The returned nodes carry
 * no reference of their own (ma_increaseRef them to keep them). This keeps the
 * loop-carried values of a while-loop resident between iterations, so each
 * iteration evaluates only its own body. Returns 0 on success. */
int ma_materialize(ma_Node **vec, int num, ma_Node **out);
/* Evaluate several nodes; async as above (scalar results always synchronise). */
int ma_evalAsync(ma_Node **vec, int num);
int ma_sync(void);
void *ma_stream(void);            /* the cudaStream_t all work is enqueued on */

void *ma_hostAlloc(size_t bytes); /* pinned host memory */
void ma_hostFree(void *p);
void *ma_devAlloc(size_t bytes);
void ma_devFree(void *p);
int ma_memcpy(void *dst, const void *src, size_t bytes, int kind); /* kind as cudaMemcpyKind */

/* Batched persistent execution: many programs (e.g. one script over hundreds
 * of rasters of uneven size) run as one persistent kernel per dependency level,
 * driven by a device work-list of (kernel kind, instance, tile) items and
 * replayed from a CUDA graph. Only Local and Focal groups can be batched; inputs
 * must be device-resident, host or file rasters; outputs go to caller device
 * buffers (16-byte aligned base and pitch).
 * ma_batchAdd returns the instance index; ma_batchPrepare fuses, autotunes tile
 * shapes (autotune != 0), compiles and captures the graph (called by the first
 * ma_batchRun when omitted); ma_batchInfo writes a JSON description.
 * ma_batchRun with sync != 0 returns non-zero when any tile reported a device
 * error (a staging wait that timed out): every output of that run is then void,
 * not only the failing tile's. */
typedef struct ma_Batch ma_Batch;
ma_Batch *ma_batchCreate(void);
int ma_batchAdd(ma_Batch *b, ma_Node **outs, int num, void **dst, const long long *pitch);
int ma_batchPrepare(ma_Batch *b, int autotune);
int ma_batchRun(ma_Batch *b, int sync);
size_t ma_batchInfo(ma_Batch *b, char *buf, size_t len);
void ma_batchDestroy(ma_Batch *b);

/* Serving over a device-resident DEM (F32, `pitch` bytes per row) with
 * continuous batching and admission by an HBM budget. Request types:
 * 0 hillshade, 1 slope, 2 viewshed (observer inside the window, height obs_h,
 * radius in cells, <= 0 for no limit), 3 D8 flow direction + flow accumulation
 * (S32 upstream counts). A request's window is an independent raster.
 * ma_serverSubmit returns the request id (-1 on error); results stay on the
 * device until ma_serverResult (copies to host and releases) or
 * ma_serverRelease. ma_serverLoad runs an open-loop Poisson load (rate req/s,
 * program mix weights mix[4], windows 256/512/1024 squared) and writes
 * latency percentiles and throughput as JSON. ma_serverCreate compiles every
 * program at the three window sizes and grows the device's stream-ordered
 * memory pool to min(budget_bytes, 4 GiB), which the pool keeps, so requests
 * allocate without waiting for the pool to map new memory. */
typedef struct ma_Server ma_Server;
ma_Server *ma_serverCreate(void *dem, long long pitch, int W, int H, size_t budget_bytes, int max_batch);
long long ma_serverSubmit(ma_Server *s, int type, int x0, int y0, int w, int h, int obs_x, int obs_y, float obs_h,
                          double radius);
int ma_serverWait(ma_Server *s, long long id, double timeout_s);
int ma_serverResult(ma_Server *s, long long id, void *dst, size_t bytes);
int ma_serverRelease(ma_Server *s, long long id);
double ma_serverLatency(ma_Server *s, long long id);
size_t ma_serverStats(ma_Server *s, char *buf, size_t len);
size_t ma_serverLoad(ma_Server *s, double rate, double seconds, const double *mix, unsigned seed, double obs_h,
                     double radius, char *buf, size_t len);
/* Closed-loop load: `outstanding` requests kept in flight for `seconds`, each
 * completion replaced at once by a new request of the mix (the throughput
 * ceiling and latency under saturation); same JSON report as ma_serverLoad. */
size_t ma_serverLoadClosed(ma_Server *s, int outstanding, double seconds, const double *mix, unsigned seed,
                           double obs_h, double radius, char *buf, size_t len);
void ma_serverDestroy(ma_Server *s);

/* Per-zone statistics (no counterpart in the reference, whose zonal skeleton
 * runtime/skeleton/ZonalSkeleton.cpp:33-292 reduces a whole raster to one
 * value): for every zone id 0 .. nzones-1 of the int32 `zone` raster, the
 * count, min, max, float32 sum and mean of the float32 `value` cells in it.
 * Cells with a zone id outside [0, nzones) or a NaN value are skipped; an empty
 * zone reports count 0, sum 0, min +inf, max -inf, mean NaN. All pointers are
 * device memory; rasters are row-major with the given pitches in bytes
 * (4-byte aligned; 16-byte aligned pointers and pitches take the vector path);
 * the outputs are arrays of nzones elements and any of them may be NULL.
 * Enqueued on `stream` (a cudaStream_t, NULL for the legacy default stream);
 * returns before the work ends. Working bins of nzones x 24 bytes come from the
 * stream's memory pool. count, min and max are exact; the sum's rounding depends
 * on the order of the device's atomic additions. */
int ma_zoneStats(const void *value, long long value_pitch, const void *zone, long long zone_pitch, int W, int H,
                 int nzones, unsigned long long *count, float *vmin, float *vmax, float *sum, float *mean,
                 void *stream);

/* ma_zoneStats without any device-memory allocation. No counterpart in the
 * reference (see ma_zoneStats). For callers that must not allocate while they
 * run: a server that reserved its whole HBM budget up front, where a pool
 * allocation could fail or exceed the budget, or a latency-critical loop,
 * where an allocation may synchronise the device or grow the memory pool.
 * The working bins are one fixed array per device in the library's own device
 * memory, so nzones may be at most 16384; larger counts return an error. Runs
 * on the calling thread's current device, checked like every other entry
 * point. The first call on a device does the set-up (loads the kernels): make
 * it before any stream capture begins. The array's address is looked up in the
 * current context on every call, so a device or context reset between calls is
 * safe, but the first call after a reset loads the kernels again (which may
 * allocate once). All calls on a device share the array: calls whose work can
 * overlap on the device (several streams or host threads) race and corrupt each
 * other's results, so order them on one stream. Same arguments, rules and
 * results as ma_zoneStats. */
int ma_zoneStatsNoAlloc(const void *value, long long value_pitch, const void *zone, long long zone_pitch, int W,
                        int H, int nzones, unsigned long long *count, float *vmin, float *vmax, float *sum,
                        float *mean, void *stream);

/* Introspection for tests and tools. */
int ma_lastLaunchCount(void);      /* kernels launched by the last evaluation */
int ma_lastGroupCount(void);       /* fusion groups of the last evaluation */
int ma_lastBandCount(void);        /* row bands of the last evaluation (0: not streamed) */
int ma_totalLaunchCount(void);
/* Fusion + code generation (+ NVRTC compilation when compile != 0) of the
 * program that evaluates `vec`, without a device. Returns the number of
 * kernels, or -1 on error. */
int ma_compileOnly(ma_Node **vec, int num, int compile);
/* Writes a text description of the fusion groups / the generated sources /
 * the plain-mode launch order into buf; returns the length needed. */
size_t ma_describeGroups(ma_Node **vec, int num, char *buf, size_t len);
size_t ma_generatedSource(ma_Node **vec, int num, char *buf, size_t len);
size_t ma_plainSchedule(ma_Node **vec, int num, char *buf, size_t len);
int ma_nodeCount(void);
void ma_collectGarbage(void);

#ifdef __cplusplus
}
#endif

#endif /* MAP_B200_H_ */
