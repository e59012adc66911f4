/*
 * nbg_b200.h — C ABI of the B200 neighbourhood-geometry library.
 *
 * The library computes, for every point of a tile, its k nearest neighbours,
 * their 3x3 covariance and its symmetric eigendecomposition, and projects the
 * result into the output dimensions of PDAL's filters.normal,
 * filters.eigenvalues and filters.covariancefeatures.  Everything runs on one
 * sm_100a GPU; there is no CPU fallback.
 *
 * Reference interfaces replaced (paths inside the PDAL fork):
 *   - filters/NormalFilter.cpp:85-182          (options, compute loop)
 *   - filters/EigenvaluesFilter.cpp:77-172     (options, filter loop)
 *   - filters/CovarianceFeaturesFilter.cpp:102-367 (options, setDimensionality)
 *   - pdal/private/KDImpl.hpp:351-381          (KD3ImplT::neighbors)
 *   - pdal/private/MathUtils.cpp:139-196,572-611 (computeCovariance, findNormal)
 *   - src/pdal/PdgNeighborhood.hpp:210-219,289-292 (fork's tryCuda*Columns seam)
 *
 * Conventions
 *   - Return codes are int: NBG_OK (0) or one of NBG_ERR_*.  The text of the
 *     last error of a context is available from nbg_last_error().
 *   - Coordinates enter as LAS-style raw int32 triples plus scale and offset;
 *     the value the reference sees is raw*scale+offset evaluated in double
 *     (pdal/pdal_types.hpp:192-193, io/private/las/Utils.cpp:527-529).
 *   - Neighbour counts include the query point (NormalFilter.cpp:135,
 *     EigenvaluesFilter.cpp:139, CovarianceFeaturesFilter.cpp:228).
 *   - Output dimensions are written as double into caller memory described
 *     by nbg_columns (base + id*point_stride + offset[d]); rows the reference
 *     skips are left untouched and reported in the row-exception list.
 */
#ifndef NBG_B200_H
#define NBG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ---------------------------------------------------- */
#define NBG_OK 0
#define NBG_ERR_INVALID 1     /* invalid argument or stage option          */
#define NBG_ERR_OOM 2         /* device allocation failed                  */
#define NBG_ERR_BUDGET 3      /* request exceeds the context's HBM budget  */
#define NBG_ERR_CUDA 4        /* CUDA runtime error                        */
#define NBG_ERR_TIMEOUT 5     /* a bounded device-side wait expired        */
#define NBG_ERR_UNSUPPORTED 6 /* input outside the supported domain        */
#define NBG_ERR_NO_DEVICE 7   /* no sm_100 device available                */
#define NBG_ERR_EXCEPTIONS 8  /* row-exception list overflowed             */

/* ---- stage kinds ----------------------------------------------------- */
#define NBG_STAGE_NORMAL 1             /* NormalX, NormalY, NormalZ, Curvature */
#define NBG_STAGE_EIGENVALUES 2        /* Eigenvalue0, Eigenvalue1, Eigenvalue2 */
#define NBG_STAGE_COVARIANCEFEATURES 3 /* selected features, bit order below */
/* Other consumers of the same kNN index (the K each queries is noted; the
 * reference's knnSearch pads a list longer than the cloud with point 0 at
 * squared distance 0, and these stages keep that):
 *   approximatecoplanar  Coplanar (0/1); K = knn, thresh1, thresh2
 *                        (ApproximateCoplanarFilter.cpp:66-114)
 *   estimaterank         Rank (0-3); K = knn, thresh1 = thresh
 *                        (EstimateRankFilter.cpp:66-84, MathUtils.cpp:197-208)
 *   nndistance           NNDistance; K = knn + 1 (knn = k), mode 0 kth / 1 avg
 *                        (NNDistanceFilter.cpp:108-138)
 *   optimalneighborhood  OptimalKNN, OptimalRadius; K = knn (= max_k), min_k
 *                        (OptimalNeighborhoodFilter.cpp:71-163)
 *   lof                  NNDistance, LocalReachabilityDistance,
 *                        LocalOutlierFactor; K = knn + 1 (knn = minpts)
 *                        (LOFFilter.cpp:66-139)
 *   outlier              Classification, written only on outlier rows and
 *                        only when some row is an inlier; mode 0 statistical
 *                        (K = knn + 1, knn = mean_k, thresh1 = multiplier) or
 *                        mode 1 radius (radius, min_k); label = class
 *                        (OutlierFilter.cpp:75-229) */
#define NBG_STAGE_APPROXIMATECOPLANAR 4
#define NBG_STAGE_ESTIMATERANK 5
#define NBG_STAGE_NNDISTANCE 6
#define NBG_STAGE_OPTIMALNEIGHBORHOOD 7
#define NBG_STAGE_LOF 8
#define NBG_STAGE_OUTLIER 9

/* covariance feature bits, in the order of feature_set "all"
 * (CovarianceFeaturesFilter.cpp:127-133) */
#define NBG_FEAT_LINEARITY (1u << 0)
#define NBG_FEAT_PLANARITY (1u << 1)
#define NBG_FEAT_SCATTERING (1u << 2)
#define NBG_FEAT_VERTICALITY (1u << 3)
#define NBG_FEAT_OMNIVARIANCE (1u << 4)
#define NBG_FEAT_ANISOTROPY (1u << 5)
#define NBG_FEAT_EIGENENTROPY (1u << 6)
#define NBG_FEAT_EIGENVALUESUM (1u << 7)
#define NBG_FEAT_SURFACEVARIATION (1u << 8)
#define NBG_FEAT_DEMANTKEVERTICALITY (1u << 9)
#define NBG_FEAT_DENSITY (1u << 10)
#define NBG_FEAT_DIMENSIONALITY 0x0Fu
#define NBG_FEAT_ALL 0x7FFu
#define NBG_NUM_FEATURES 11

/* eigenvalue modes (CovarianceFeaturesFilter.cpp:71-86) */
#define NBG_MODE_RAW 0
#define NBG_MODE_SQRT 1
#define NBG_MODE_NORMALIZED 2

/* per-row exception codes; the stage shim turns them into the reference's
 * log lines or exceptions */
#define NBG_ROW_TOO_FEW 1       /* findNormal: fewer than 3 neighbours        */
#define NBG_ROW_ZERO_COV 2      /* covariance isZero() (|b_ij| <= 1e-12)      */
#define NBG_ROW_EIGEN_FAIL 3    /* eigensolver reported failure               */
#define NBG_ROW_ZERO_LAMBDA 4   /* covariancefeatures: largest eigenvalue 0   */
#define NBG_ROW_RADIUS_FEW 5    /* radius search found fewer than min_k points;
                                   `reserved` holds the count (capped at 65535) */

#define NBG_MAX_DIMS 16

/* Options of one stage, same names and meaning as the reference's
 * ProgramArgs (NormalFilter.cpp:85-97, EigenvaluesFilter.cpp:77-87,
 * CovarianceFeaturesFilter.cpp:102-113).  `knn` is the user's value; the
 * library adds the query point itself. */
typedef struct nbg_stage_opts {
    int32_t kind;          /* NBG_STAGE_*                                    */
    int32_t knn;           /* k nearest neighbours, excluding the point      */
    int32_t always_up;     /* normal: flip so that NormalZ >= 0              */
    int32_t has_viewpoint; /* normal: orient towards viewpoint[]             */
    double viewpoint[3];
    int32_t refine;        /* normal: accepted; output-neutral in the
                              reference (NormalFilter.cpp:184-286 refines a
                              copy of the normal)                            */
    int32_t normalize;     /* eigenvalues: divide by their sum               */
    uint32_t feature_mask; /* covariancefeatures: NBG_FEAT_* bits            */
    int32_t mode;          /* covariancefeatures: NBG_MODE_*; nndistance: 0 kth,
                              1 avg; outlier: 0 statistical, 1 radius,
                              2 unrecognised method (the stage is a no-op)   */
    int32_t stride;        /* keep every stride-th of knn*stride neighbours  */
    int32_t optimized;     /* covariancefeatures: per-point k = OptimalKNN   */
    int32_t use_radius;    /* neighbours = the points within `radius` (squared
                              FP64 distance < radius*radius) instead of knn
                              (KDImpl.hpp:398-415)                           */
    int32_t min_k;         /* eigenvalues/covariancefeatures with a radius:
                              rows with fewer neighbours are skipped;
                              optimalneighborhood: smallest k; outlier
                              (radius): inliers have more than min_k         */
    double radius;
    double thresh1;        /* approximatecoplanar thresh1, estimaterank
                              thresh, outlier multiplier                     */
    double thresh2;        /* approximatecoplanar thresh2                    */
    int32_t label;         /* outlier: class written to outlier rows         */
    int32_t eigen_fp64;    /* 1: every row of the stage's neighbourhood group
                              is solved by the FP64 Eigen chain alone (a plain
                              FP64 eigensolve); 0: FP32 Jacobi + FP64 polish,
                              the chain only where the polish does not settle
                              or a sign needs it.  Both meet the same bars.  */
} nbg_stage_opts;

/* Output placement: dimension d of point id is the double at
 *   (char*)base + id*point_stride + offset[d].
 * A PDAL row layout is point_stride = record size; a column layout is
 * point_stride = 8 and offset[d] = d*n*8. */
typedef struct nbg_columns {
    void* base;
    int64_t point_stride;
    int32_t ndims;
    int32_t on_device;     /* 1: base is device memory; 0: host memory whose
                              skipped rows keep their values; 2: host memory of
                              freshly added dimensions (skipped rows read 0) */
    int64_t offset[NBG_MAX_DIMS];
} nbg_columns;

/* One row the reference would skip or reject. */
typedef struct nbg_row_exception {
    uint32_t point_id;
    uint8_t stage;         /* index into the stage array of the call         */
    uint8_t code;          /* NBG_ROW_*                                      */
    uint16_t reserved;
} nbg_row_exception;

/* Per-call counters (filled by nbg_run when non-null). */
typedef struct nbg_run_stats {
    uint64_t points;          /* queries answered                               */
    uint64_t tie_rows;        /* rows whose k-th boundary tied: ordered on the
                                 KD replica's tree                              */
    uint64_t deferred_rows;   /* rows the ring search could not finish          */
    uint64_t resolved_rows;   /* rows whose eigenproblem the FP32 solver handed
                                 to the FP64 chain (near-degenerate spectra)    */
    double grid_ms;           /* device time of the grid build                  */
    double query_ms;          /* device time of the fused query kernel(s)       */
    double tree_ms;           /* device time after the query kernel: KD replica
                                 build (when not overlapped), tie ordering and
                                 search replay                                  */
    double total_ms;          /* device time of the whole call                  */
    uint64_t kernel_launches; /* device kernels this library launched in the call */
    uint64_t replay_rows;     /* rows answered by the full nanoflann search replay
                                 (deferred rows, tie groups over 32 points)     */
    double kd_build_ms;       /* device time of the KD replica build on the side
                                 stream, overlapped with the query kernel       */
    uint64_t outliers;        /* outlier stages: rows found to be outliers
                                 (written only when inliers remain)             */
    uint64_t inliers;         /* outlier stages: rows found to be inliers       */
    uint64_t output_chunks;   /* host records copied back in this many chunks of
                                 the point-id range, each while the later chunks
                                 were answered (0: one copy at the end)         */
    uint64_t retry_rows;      /* rows a faster select kernel handed to the
                                 two-pass ring search (nbg_tile_set_select)     */
} nbg_run_stats;

typedef struct nbg_context nbg_context;
typedef struct nbg_tile nbg_tile;

/* Library and device ------------------------------------------------------ */
const char* nbg_version(void);
int nbg_device_count(void);

/* Context: owns device scratch, resident tiles and the HBM budget.
 * Replaces the fork's resident neighbourhood lifetime
 * (src/pdal/PdgNeighborhood.cpp:1383-1550).
 * Threads: the calls that take a context serialise on it (uploads, runs,
 * tuning and frees of its tiles wait for one another), so a context may be
 * shared; for work that overlaps on the GPU use one context per thread, or
 * the served form below, whose slots each own one.  nbg_last_error reports
 * the context's most recent failure, whichever thread made it. */
int nbg_create(nbg_context** ctx, int device, uint64_t hbm_budget_bytes);
int nbg_destroy(nbg_context* ctx);
const char* nbg_last_error(const nbg_context* ctx);

/* Tile: a point set with its uniform grid, resident on the device.
 * x/y/z are raw int32 coordinates (host or device memory, `on_device`).
 * Replaces PointView::build3dIndex (pdal/PointView.cpp:264-290) and the
 * fork's SpatialIndex::build (src/index/SpatialIndexKernels.cu:1772-1906). */
int nbg_tile_upload(nbg_context* ctx, const int32_t* x, const int32_t* y,
                    const int32_t* z, uint64_t n, const double scale[3],
                    const double offset[3], int32_t on_device, void* stream,
                    nbg_tile** tile);
int nbg_tile_free(nbg_context* ctx, nbg_tile* tile);

/* Grid tuning of a tile: the cell edge is ceil(cell_factor * r_k), r_k the
 * radius holding k points at the tile's planar density (default factor 4);
 * fixed_cell > 0 forces an edge in raw units.  Takes effect at the next run
 * (the grid is rebuilt).  Used by the autotuner; no counterpart in the
 * reference (whose KD tree has no tunable). */
int nbg_tile_tune(nbg_context* ctx, nbg_tile* tile, float cell_factor, int32_t fixed_cell);
/* Select kernel of a tile (the k-nearest search of nbg_run; results are
 * identical for every setting):
 *   0  two-pass ring search, one query per thread (default)
 *   1  the same with the queries of each 256-row block in Morton order
 *   2  single-pass ring search: top-list keys carry the candidate's column and
 *      position, so the K nearest are read back without a second scan
 *   8, 16, 32  that many neighbouring queries (Morton-compact) share one
 *      candidate list, gathered box ring by box ring from a first margin of
 *      first_margin cell edges
 * Rows the faster forms cannot answer exactly go to the two-pass search.
 * Used by the autotuner; no counterpart in the reference. */
int nbg_tile_set_select(nbg_context* ctx, nbg_tile* tile, int32_t select_kernel,
                        float first_margin);
/* Autotuner: builds the tile's grid with each candidate cell factor (null:
 * 1, 1.5, 2, 3, 4, 6), times the select pass (best of three launches) on one
 * contiguous window of the tile's rows in grid order (the whole tile up to 8M
 * rows), and keeps the factor with the least estimated grid + query time
 * (rows the ring search would defer charged at 5 us each).  For each factor it also
 * times the select kernels of nbg_tile_set_select (0, 1, 2 and 32)
 * on the same sample rows, select + finish, and keeps the fastest pair.  The
 * choice is cached per (log2 points, neighbour slots) class of the context;
 * with use_cache a cached class is applied without measuring.  nbg_run applies
 * the cached choice of a tile's class to every tile whose cell factor and
 * select kernel the caller left alone (no nbg_tile_tune, nbg_tile_set_select
 * or nbg_tile_autotune on it), so a loaded tuning file reaches fresh tiles. */
int nbg_tile_autotune(nbg_context* ctx, nbg_tile* tile, int32_t knn, const float* candidates,
                      int32_t n_candidates, int32_t use_cache, float* chosen, void* stream);

/* The autotuner's cached choices, to keep them in a tuning file across
 * processes: one entry per (log2 points, neighbour slots) class.
 * nbg_autotune_cache_get writes up to `capacity` entries (sorted by class)
 * and the number the cache holds to *count; nbg_autotune_cache_set adds or
 * replaces entries (NBG_ERR_INVALID for a class outside [0, 63] x [1, 128],
 * a factor that is not finite and positive, or a select kernel other than
 * 0, 1, 2, 8, 16, 32; nothing is set then). */
typedef struct nbg_tune_entry {
    int32_t size_class;    /* floor(log2(points))                            */
    int32_t slots;         /* neighbour slots of the select kernel           */
    float cell_factor;
    int32_t select_kernel;     /* nbg_tile_set_select                        */
} nbg_tune_entry;
int nbg_autotune_cache_get(nbg_context* ctx, nbg_tune_entry* entries, int32_t capacity,
                           int32_t* count);
int nbg_autotune_cache_set(nbg_context* ctx, const nbg_tune_entry* entries, int32_t count);
uint64_t nbg_tile_size(const nbg_tile* tile);

/* Run stages over a resident tile.  Stages sharing knn share one fused
 * kNN + covariance + eigen pass.  `optimal_knn`/`optimal_radius` are the
 * per-point OptimalKNN / OptimalRadius input columns (double, indexed by
 * point id, host or device per `aux_on_device`), needed only for the
 * Density feature and for `optimized`.  Replaces the per-point loops at
 * NormalFilter.cpp:140-182, EigenvaluesFilter.cpp:115-172 and
 * CovarianceFeaturesFilter.cpp:175-367. */
int nbg_run(nbg_context* ctx, nbg_tile* tile, const nbg_stage_opts* stages,
            int32_t n_stages, const nbg_columns* outputs,
            const double* optimal_knn, const double* optimal_radius,
            int32_t aux_on_device, nbg_row_exception* exceptions,
            uint32_t exception_capacity, uint32_t* n_exceptions,
            nbg_run_stats* stats, void* stream);

/* Neighbour ids of every point (sorted ascending per row, `rows` x `k1`
 * uint32, k1 = min(knn+1, n)), for parity checks against KD3Index. */
int nbg_neighbor_sets(nbg_context* ctx, nbg_tile* tile, int32_t knn,
                      uint32_t* ids_out, int32_t ids_on_device,
                      nbg_run_stats* stats, void* stream);

/* LAS ingest -------------------------------------------------------------
 * The fields of a LAS 1.0-1.4 public header block the path needs, and a tile
 * made straight from the file's point records: the records (host or device
 * memory, record_length bytes each, X/Y/Z int32 at their start as in every
 * point format 0-10) are decoded on the device, so coordinates enter as the
 * file's own raw integers with its scale and offset.  Replaces the reader
 * step of the fork's device LAS path (src/io/las/LasKernels.cu:266-321,
 * src/pdal/PdgNeighborhood.cpp:1115-1192).  LAZ (compressed) records are not
 * decoded here: nbg_las_header reports them in `compressed`. */
typedef struct nbg_las_info {
    uint8_t version_major;
    uint8_t version_minor;
    uint8_t point_format;         /* 0-10                                   */
    uint8_t compressed;           /* LAZ: records are not plain LAS records  */
    uint16_t point_record_length;
    uint16_t reserved;
    uint32_t offset_to_points;    /* byte offset of the first record         */
    uint64_t point_count;
    double scale[3];
    double offset[3];
    double min[3];
    double max[3];
} nbg_las_info;
int nbg_las_header(const void* bytes, size_t size, nbg_las_info* info);
int nbg_tile_upload_las(nbg_context* ctx, const void* records, uint64_t n,
                        uint32_t record_length, int32_t on_device, const double scale[3],
                        const double offset[3], void* stream, nbg_tile** tile);

/* Stage layer ------------------------------------------------------------
 * PDAL pipeline JSON and the stage logic above nbg_run, so an existing
 * pipeline is a drop-in.  nbg_filter_create parses one stage's options
 * object as ProgramArgs would (NormalFilter.cpp:85-97, EigenvaluesFilter.cpp:
 * 77-87, CovarianceFeaturesFilter.cpp:102-113, and the other consumers' addArgs
 * listed with their stage kinds above; value errors as ProgramArgs.hpp:
 * 415-435), registers its dimensions (addDimensions) and runs prepared()'s
 * checks; has_optimal_knn / has_optimal_radius say whether the input view
 * carries those dimensions.  A check the reference throws from returns
 * NBG_ERR_INVALID with "<stage>: <the reference's message>" in err. */
typedef struct nbg_filter nbg_filter;
int nbg_filter_create(const char* type, const char* options_json, int32_t has_optimal_knn,
                      int32_t has_optimal_radius, nbg_filter** filter, char* err, size_t err_len);
/* The stage's nbg_stage_opts (knn as the user gave it; with a radius,
 * use_radius/radius/min_k set).  NBG_ERR_UNSUPPORTED (with *out still
 * filled) when stride * (knn + 1) exceeds 65. */
int nbg_filter_options(const nbg_filter* filter, nbg_stage_opts* out);
/* Registered output dimensions, comma separated, in the library's order. */
int nbg_filter_dims(const nbg_filter* filter, char* names, size_t len);
/* Lines the stage logged (prepared() warnings, then per-row skip lines). */
const char* nbg_filter_log(const nbg_filter* filter);
/* The reference's reaction to a run's row exceptions for this stage (its
 * index in the nbg_run call): Info lines appended to the log in point order,
 * or NBG_ERR_INVALID with the text its loop would throw. */
int nbg_filter_report(nbg_filter* filter, const nbg_row_exception* exceptions, uint32_t n,
                      int32_t stage_index, char* err, size_t err_len);
/* filters.outlier's warnings after a run (OutlierFilter.cpp:191-226):
 * "would remove all points" when no row is an inlier, "no outliers" when no
 * row is an outlier; appended to the log.  No-op for the other stages. */
int nbg_filter_outcome(nbg_filter* filter, const nbg_run_stats* stats);
void nbg_filter_free(nbg_filter* filter);

/* A pipeline JSON (an array of stages, or {"pipeline": [...]}): its stages'
 * types ("file" for a bare file name) and option objects as JSON text. */
typedef struct nbg_pipeline nbg_pipeline;
int nbg_pipeline_parse(const char* json, nbg_pipeline** pipeline, char* err, size_t err_len);
int32_t nbg_pipeline_size(const nbg_pipeline* pipeline);
const char* nbg_pipeline_type(const nbg_pipeline* pipeline, int32_t index);
const char* nbg_pipeline_options(const nbg_pipeline* pipeline, int32_t index);
void nbg_pipeline_free(nbg_pipeline* pipeline);

/* Batched form -----------------------------------------------------------
 * Many tiles of uneven size and knn in one call: the tiles' grids are built,
 * then one persistent kernel per neighbour-count class drains a device work
 * queue of (tile, 128-query block) items and one more finishes every row,
 * all captured in a CUDA graph (replayed while the batch's shape is
 * unchanged); the KD replicas for tie rows are built on a side stream while
 * the queue drains.  Each item's results equal those of nbg_run on that
 * tile.  Outputs, OptimalKNN/OptimalRadius and the tiles are device-resident;
 * the stages of one item share one knn; a tile appears at most once. */
typedef struct nbg_batch_item {
    nbg_tile* tile;
    int32_t n_stages;
    uint32_t exception_capacity;
    const nbg_stage_opts* stages;
    const nbg_columns* outputs;       /* on_device = 1                       */
    const double* optimal_knn;        /* device, may be null                 */
    const double* optimal_radius;
    nbg_row_exception* exceptions;    /* host, exception_capacity entries    */
    uint32_t* n_exceptions;           /* host, may be null                   */
} nbg_batch_item;

#define NBG_BATCH_GRAPH 1u            /* capture the queue launches in a graph */
#define NBG_BATCH_AUTOTUNE 2u         /* cell factor per tile from the autotuner
                                         (cached per size/knn class)          */

int nbg_run_batch(nbg_context* ctx, const nbg_batch_item* items, int32_t n_items,
                  uint32_t flags, nbg_run_stats* stats, void* stream);

/* Served form ------------------------------------------------------------
 * A request loop over one device: requests (one tile + its stages each) are
 * queued FIFO and admitted while a slot is free and the HBM budget holds the
 * request's estimated footprint; each slot is a host worker with its own
 * context and stream, so admitted requests overlap on the device (continuous
 * batching: a request that arrives while others run starts as soon as a slot
 * and memory free up).  The reference has no counterpart (its stages run one
 * view at a time, pdal/Stage.hpp:419-497); each request does exactly what
 * nbg_tile_upload + nbg_run + nbg_tile_free do, so results are the same
 * alone and in any mix.  The caller's buffers must stay valid until the
 * request completes. */
typedef struct nbg_request {
    const int32_t* x;            /* raw coordinates, caller order           */
    const int32_t* y;
    const int32_t* z;
    uint64_t n;
    double scale[3];
    double offset[3];
    int32_t on_device;           /* x/y/z are device pointers               */
    int32_t n_stages;
    const nbg_stage_opts* stages;
    const nbg_columns* outputs;  /* one per stage, as nbg_run               */
    const double* optimal_knn;   /* may be null                             */
    const double* optimal_radius;
    int32_t aux_on_device;
    uint32_t exception_capacity;
    nbg_row_exception* exceptions;
    uint64_t user_tag;
} nbg_request;

typedef struct nbg_request_result {
    int32_t status;              /* NBG_OK or the run's error code          */
    uint32_t n_exceptions;
    uint64_t user_tag;
    double submit_us;            /* host clock, microseconds since creation */
    double start_us;             /* admitted to a slot                      */
    double end_us;               /* results in the caller's buffers         */
    uint64_t est_bytes;          /* footprint the admission charged         */
    nbg_run_stats stats;
} nbg_request_result;

typedef struct nbg_server nbg_server;

/* slots: concurrent requests (host workers); hbm_budget_bytes 0 = no limit */
int nbg_server_create(nbg_server** server, int32_t device, int32_t slots,
                      uint64_t hbm_budget_bytes);
/* Queues a request; *ticket identifies it.  NBG_ERR_BUDGET when the request
 * alone exceeds the budget. */
int nbg_server_submit(nbg_server* server, const nbg_request* request, uint64_t* ticket);
/* Waits up to timeout_ms (< 0: no limit) for a request; NBG_ERR_TIMEOUT if
 * it has not finished.  A finished request's result is returned once. */
int nbg_server_wait(nbg_server* server, uint64_t ticket, int32_t timeout_ms,
                    nbg_request_result* result);
/* Estimated device footprint of a request (what admission charges). */
uint64_t nbg_request_bytes(const nbg_request* request);
const char* nbg_server_last_error(const nbg_server* server);
/* Waits for every queued request, then stops the workers. */
int nbg_server_destroy(nbg_server* server);

/* No-allocation entry point.  This function has no counterpart in the
 * reference; it exists for callers that cannot allocate device memory when
 * they need results: code running inside another framework's allocator or
 * memory pool, real-time loops that must not call cudaMalloc/cudaFree, and
 * plug-in hosts that forbid allocation in their processing callbacks.
 *
 * Runs one stage over one tile of at most NBG_NOALLOC_MAX_POINTS points.
 * x/y/z, outputs (on_device must be 1), `unresolved` (capacity n),
 * `exceptions`, `optimal_knn`/`optimal_radius` are device memory owned by the
 * caller; n_unresolved / n_exceptions are host pointers.  All working memory
 * (grid, scan storage, counters: about 49 MB) is one fixed device
 * array inside this library, present on every GPU that loads it until the
 * process exits; nothing is allocated or freed.  Larger tiles, and tiles
 * whose columns span more cells than the fixed table holds (4 per point),
 * are rejected with NBG_ERR_UNSUPPORTED and a message in err_msg (caller
 * buffer, may be null).
 *
 * Rows whose neighbour set depends on the reference's tie order (or whose
 * ring search did not finish) need the exact KD replica, whose memory grows
 * with the tile; their point ids are written to `unresolved` and their
 * outputs are left untouched, so the caller can answer them with nbg_run.
 * Every other row equals what nbg_run writes.
 *
 * The first call on each device looks up the array's device address; make
 * that first call outside any stream capture.  Every call shares the array:
 * calls whose work overlaps on one device race. */
#define NBG_NOALLOC_MAX_POINTS 524288u
int nbg_stage_noalloc(const int32_t* x, const int32_t* y, const int32_t* z, uint64_t n,
                      const double scale[3], const double offset[3],
                      const nbg_stage_opts* opts, const nbg_columns* out,
                      const double* optimal_knn, const double* optimal_radius,
                      uint32_t* unresolved, uint32_t* n_unresolved,
                      nbg_row_exception* exceptions, uint32_t exception_capacity,
                      uint32_t* n_exceptions, void* stream, char* err_msg, size_t err_len);

/* Diagnostic: the device replica of the reference's KD tree for a tile
 * (built on demand): point order `vind` (n ids) and up to `node_capacity`
 * nodes (child ids or -1, cut dim, divlow, divhigh, vind range).  Mirrors
 * nanoflann's tree (vendor/nanoflann/nanoflann.hpp:640-873) for parity
 * tests; not needed for normal use. */
int nbg_debug_kd_export(nbg_context* ctx, nbg_tile* tile, uint32_t* vind, uint32_t* n_nodes,
                        int32_t* child1, int32_t* child2, int32_t* divfeat, double* divlow,
                        double* divhigh, uint32_t* begin, uint32_t* end,
                        uint32_t node_capacity);

#ifdef __cplusplus
}
#endif
#endif /* NBG_B200_H */
