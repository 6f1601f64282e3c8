/*
 * livox_b200.h -- C ABI of the B200 (sm_100a) per-frame LiDAR SLAM hot path.
 *
 * Every entry point is `extern "C"`, takes plain device pointers, sizes and a cudaStream_t passed as
 * `void*`, enqueues its kernels on that stream and returns an int status:
 *     LW_OK (0), LW_EINVAL (bad argument), LW_ECAPACITY (a capacity is exceeded),
 *     LW_ETIMEOUT (a bounded device wait gave up), LW_ECUDA (a CUDA call failed).
 * lw_last_error() returns a message for the calling thread's last failure.
 * The library never allocates device memory: the caller (the Python `livox_warp` package, or any other
 * host) allocates every buffer and passes pointers and capacities.
 *
 * Conventions shared with the reference implementation (python/livox_warp in nhaumann/livox-warp):
 *   - voxel keys pack three 21-bit biased axis indices into an int64 (gpu.py:231-239), -1 is an empty slot;
 *   - slot hash = (key * 0x9E3779B97F4A7C15) ^ (>> 29 arithmetic), & 0x7FFFFFFF, & mask (gpu.py:247-251);
 *   - open addressing with at most 64 linear probes (gpu.py:254-265);
 *   - attr packs reflectivity (bits 0-7), noise tag (8-15), return index (16-23), device (24-31)
 *     (sources.py:1-9).
 * Deviations, all chosen so that the GPU path is deterministic and matches the CPU oracle bit for bit:
 *   - per-voxel sums are exact int64 fixed point (LW_FIX_* units) instead of float32 atomics of
 *     undefined order; means and covariances are derived from them in float64;
 *   - "the first thread to claim" becomes "the lowest point index", and the 4096-point caps take the
 *     first points in index order.
 */
#ifndef LIVOX_B200_H
#define LIVOX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------------- */
#define LW_OK 0
#define LW_EINVAL (-1)
#define LW_ECAPACITY (-2)
#define LW_ETIMEOUT (-3)
#define LW_ECUDA (-4)

/* ---- fixed-point units of the voxel sums ------------------------------------------------------ */
#define LW_FIX_R 4294967296.0        /* registration map: units per metre of (point - voxel centre), 2^32 */
#define LW_FIX_RR 1099511627776.0    /* registration map: units per m^2 of the outer products, 2^40 */
#define LW_FIX_W 1048576.0           /* integration / cluster maps: units per metre of world xyz, 2^20 */
#define LW_REG_CAP 4096              /* points a registration voxel sums (odom.py:83) */
#define LW_MAP_CAP 4096              /* points an integration voxel sums (gpu.py:55) */
#define LW_ACC_STRIDE 64             /* entries of one Gauss-Newton accumulator (odom.py:72-82) */
#define LW_GN_TRACE 17               /* poses a Gauss-Newton trace holds: the start and up to 16 iterations */
#define LW_REC_FLOATS 20             /* floats of a registration voxel's derived record */
#define LW_POSE_SLOTS 65536          /* pose table entries (gpu.py:56) */

/* accumulator layout (odom.py:74-82; localize.py shares it) */
#define LW_ACC_H 0
#define LW_ACC_B 21
#define LW_ACC_COUNT 27
#define LW_ACC_ERR 28
#define LW_ACC_RMS 29
#define LW_ACC_WEIGHT 30
#define LW_ACC_RANGE 31
#define LW_ACC_HG 32

/* ---- library ---------------------------------------------------------------------------------- */
const char* lw_version(void);
const char* lw_last_error(void);
/* Number of SMs of the current device (the persistent kernels launch one CTA per SM). */
int lw_device_sms(int* out_sms);

/* Opt-in launch timing: when enabled, the entry points bracket their main kernels with CUDA events on the
 * launching stream ("gn", "thin", "reg_insert", "map_insert", "carve", "frame_append", "control", "map_build");
 * lw_prof_read waits for them and returns the summed milliseconds and the launch count of one name. */
int lw_prof_enable(int on);
int lw_prof_read(const char* name, double* ms, int64_t* count);
int lw_prof_reset(void);
/* Kernels this library has launched since the last reset (reset when `reset` is non-zero). */
int64_t lw_launches(int reset);

/* ---- registration voxel map (odom.py:468-474) -------------------------------------------------- */
typedef struct lw_regmap {
    int64_t* keys;   /* [cap] voxel key or -1 */
    int32_t* cnt;    /* [cap] points summed into the voxel (<= LW_REG_CAP) */
    int64_t* sum;    /* [cap*3] sum of (w - voxel centre), LW_FIX_R units */
    int64_t* outer;  /* [cap*6] sum of (w - c)(w - c)^T upper triangle xx,xy,xz,yy,yz,zz, LW_FIX_RR units */
    float* rec;      /* [cap*LW_REC_FLOATS] derived record: mean(3), count, M(6), Mg(6), q(3), surface */
    int32_t* bcnt;   /* [cap] scratch, 0 between calls */
    int32_t* first;  /* [cap] scratch, INT32_MAX between calls */
    int32_t* stats;  /* [2] voxels claimed, points that found no slot in the probe window */
    int64_t cap;     /* slots, a power of two; at most 2^25 for the Gauss-Newton entry points */
} lw_regmap;

/* What a registration voxel's record is derived with (odom.py:337-368, 759-761). */
typedef struct lw_rec_params {
    float voxel;   /* registration voxel (m) */
    float tight2;  /* (TIGHT_FRACTION * voxel / sqrt(12))^2 */
    float noise2;  /* sensor range noise variance */
    float alpha;   /* weight of loose directions */
} lw_rec_params;

/* ---- odometry (odom.py:458-803) --------------------------------------------------------------- */
typedef struct lw_odom_params {
    double frame_dt, reg_voxel, min_range, max_range, noise, alpha, damping, velocity_smooth;
    double degen_thr, prior_info, kf_dist, kf_angle_deg;
    int32_t max_iter, warmup, min_points, min_corr, ret_mask, deskew, redeskew, frame_cap;
} lw_odom_params;

/* Device-resident odometry state; the host reads it back only when it asks for stats or poses. */
typedef struct lw_odom_state {
    double T[16];       /* pose of the last finalised frame (sensor to world, row major) */
    double T_prev[16];
    double T_key[16];   /* pose of the last keyframe */
    double delta[16];   /* constant-velocity motion per frame */
    double xi_s[6];     /* smoothed body twist */
    double T_pred[16];  /* the current registration's start / prior pose */
    double T_reg[16];   /* the current registration's result */
    double t_mid;       /* mid-frame time of the frame being finalised */
    double rms, cond;   /* stats of the last registration */
    float xi[6];        /* body twist of the last frame (rho, theta), what deskew uses */
    float xi_used[6];   /* twist the current frame was deskewed with */
    int32_t has_prev, has_key, map_frames, frame_k;
    int32_t m, n_ds, warm, ok;
    int32_t run_reg, do_insert, redo, err;
    int32_t iters, corr, degen, weak;
    int32_t frames, skipped, keyframes, traj_len;
    int32_t iters_first, pad_; /* Gauss-Newton iterations of the frame's first registration (from the prediction) */
} lw_odom_state;

/* One finalised frame in the device trajectory log. */
typedef struct lw_traj_rec {
    double T[16];
    double t_mid;
    int32_t k, ok, iters, corr;
    int32_t iters_first, pad_; /* iterations of the first registration; iters is the last one's */
} lw_traj_rec;

/* Frame buffers owned by Odometry (odom.py:476-490). */
typedef struct lw_frame_buf {
    float* f_raw;     /* [cap*4] x, y, z, t as measured */
    float* f_xyz;     /* [cap*4] x, y, z (deskewed to mid-frame), t */
    uint32_t* f_attr; /* [cap] */
    float* f_t;       /* [cap] */
    int32_t* f_frame; /* [cap] */
    int32_t* count;   /* [1] points in the open frame (may exceed cap: the excess is dropped) */
    int64_t* ds_keys; /* [ds_cap] thinning table, -1 between frames */
    int32_t* ds_win;  /* [ds_cap] lowest point index per thinning voxel, INT32_MAX between frames */
    int32_t* ds_slot; /* [cap] per point: its thinning slot when kept, else -1 */
    int32_t* tiles;   /* [cap/1024 + 1] per-tile kept counts */
    float* ds_xyz;    /* [cap*4] thinned points x, y, z, range */
    int64_t cap;      /* frame capacity */
    int64_t ds_cap;   /* thinning slots, a power of two >= cap */
} lw_frame_buf;

/* Scratch of the persistent Gauss-Newton kernel. */
typedef struct lw_gn_scratch {
    double* part;      /* [2 * grid * LW_ACC_STRIDE] per-CTA partials (lw_icp_accumulate); the Gauss-Newton loop's
                          fixed-point sums and the thinning's per-CTA counts (grid >= 2) */
    uint32_t* bar;     /* [2] grid barrier count and exit count; zero before the first launch, and every launch
                          leaves both zero */
    int32_t* err;      /* [1] set when a bounded wait gives up (1) or a fixed-point sum overflows (4); sticky */
    int32_t grid;      /* CTAs (2 .. the SM count, one per SM) */
    int32_t spin_budget; /* barrier wait limit in polls (~0.1-0.3 us each); 0 = the default (2^24 polls) */
    int32_t skip_cta;  /* failure injection for tests of the bounded wait: this CTA leaves before the first
                          barrier, so the others time out and the launch reports err = 1; -1 = none */
    double* trace;     /* NULL, or [LW_GN_TRACE * 12]: the start pose and the pose after each iteration (the top
                          3 rows of the 4x4, row major), for studies of how fast a registration converges */
} lw_gn_scratch;

/* Pose table of the Pipeline (gpu.py:1196-1206); written on the device by the odometry. */
typedef struct lw_pose_table {
    float* poses;         /* [LW_POSE_SLOTS*16] row-major sensor-to-world */
    float* tw;            /* [LW_POSE_SLOTS*6] rho, theta per frame */
    int32_t* owner_frame; /* [LW_POSE_SLOTS] */
    int32_t* owner_epoch; /* [LW_POSE_SLOTS] */
} lw_pose_table;

/* Append the staged points with k_min <= floor(max(t,0)/frame_dt) <= k_open to the open frame, in
 * staged order (odom.py:97-123, called from Odometry.push odom.py:626-638). xyz is [n*xyz_stride]. */
int lw_frame_append(const float* xyz, int32_t xyz_stride, const uint32_t* attr, const float* t, int64_t n,
                    double inv_dt, int32_t k_min, int32_t k_open, lw_frame_buf* fb, void* stream);

/* Zero the open frame's point count (odom.py:614, 636). */
int lw_frame_reset(lw_frame_buf* fb, void* stream);

/* Finalise the open frame k (odom.py:642-657 with _estimate :659-680, _register :752-803, _insert :719,
 * _update_velocity :682): deskew, thin, Gauss-Newton on the device, re-deskew and re-register when the
 * solved motion differs, keyframe insert, velocity update, pose-table entry and trajectory record.
 * `m_ub` bounds the frame's point count (grid sizing only). No host synchronisation. */
int lw_odom_finalize(int32_t k, int64_t m_ub, const lw_odom_params* prm, lw_odom_state* st, lw_frame_buf* fb,
                     lw_regmap* reg, lw_gn_scratch* gn, lw_pose_table* pt, int32_t epoch,
                     lw_traj_rec* traj, int64_t traj_cap, void* stream);

/* Write a pose and twist for frames k0 .. k1-1 into the pose table (odom.py:615-625, 637): what the live
 * view draws frames with before they are solved. mode bit 0: the current pose T instead of the prediction
 * T*delta; bit 1: a zero twist instead of xi. */
int lw_odom_predict_poses(int32_t k0, int32_t k1, int32_t current, const lw_odom_state* st, lw_pose_table* pt,
                          int32_t epoch, void* stream);

/* Reset the odometry state to pose T0 (odom.py:561-579) and, when `clear_map`, the registration map. */
int lw_odom_reset(const double* T0_host, lw_odom_state* st, lw_regmap* reg, int32_t clear_map, void* stream);

/* Forget the frame clock only (odom.py:581-589). */
int lw_odom_restart_clock(lw_odom_state* st, void* stream);

/* ---- the parts of the frame, exposed one by one ------------------------------------------------ */

/* Deskew m points (odom.py:163-178, gpu.py:268-283): s = clamp((t - t_mid) * inv_dt, -1, 1),
 * p' = rotvec(theta s) p + rho s. raw and out are [m*4] (x, y, z, t); m is a device count. */
int lw_deskew(const float* raw, float* out, const int32_t* m_dev, int64_t m_ub, double t_mid, double inv_dt,
              const float* twist6_host, void* stream);

/* Thin the deskewed frame: keep the lowest-index point of every half-voxel (odom.py:126-160, 731-737);
 * writes fb->ds_xyz in point order and n_ds_dev. */
int lw_thin(lw_frame_buf* fb, const int32_t* m_dev, int64_t m_ub, double inv_v, double min_range,
            double max_range, int32_t ret_mask, int32_t* n_ds_dev, void* stream);

/* Thinning for callers that cannot allocate device memory; it has no counterpart in the reference.
 * A real-time sensor thread, or a host whose device memory is fixed at start-up (a driver callback, a plugin
 * under a memory budget), must not call cudaMalloc on the frame path: an allocation can wait behind other
 * device work for an unbounded time. This variant of lw_thin takes only the caller's points (xyz4 [m*4] with
 * x, y, z, any; attr [m]) and output (ds4_out [m*4], *n_ds_dev); its tables live in one file-scope device
 * array of about 1.8 MB that every GPU which loads the library holds until the process exits. At most 65536
 * points per call: more is rejected with LW_ECAPACITY before any work is queued. The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. It allocates nothing. Calls share the one array and each clears its tables
 * first, so calls that overlap on the GPU (two streams at once) race: serialise them. xyz4 and ds4_out must
 * be 16-byte aligned (LW_EINVAL otherwise). The array's address is looked up once per device and kept: after
 * a cudaDeviceReset of a device, do not call it on that device again in the same process. */
int lw_thin_noalloc(const float* xyz4, const uint32_t* attr, int64_t m, double inv_v, double min_range,
                    double max_range, int32_t ret_mask, float* ds4_out, int32_t* n_ds_dev, void* stream);

/* Add n points posed by T to the registration map (odom.py:186-230) and refresh the derived record of
 * every voxel touched. xyz is [n*4]; n_dev is a device count or NULL (then n_ub is the count);
 * pslot is [n_ub] scratch. */
int lw_reg_insert(const float* xyz4, const uint32_t* attr, const int32_t* n_dev, int64_t n_ub,
                  const double* T_host, double voxel, double max_range, int32_t ret_mask, lw_regmap* reg,
                  const lw_rec_params* rp, int32_t* pslot, void* stream);

/* Recompute every occupied voxel's record (after the record parameters change). */
int lw_reg_refresh_all(lw_regmap* reg, const lw_rec_params* rp, void* stream);

/* One Gauss-Newton accumulation pass (odom.py:275-375 then k_reduce :378-384) at pose T: out[64] in the
 * LW_ACC_* layout (float64). reach / max_d2 / kappa as odom.py:765-767. The Jacobian is taken about the
 * world origin, as the reference does. */
int lw_icp_accumulate(const float* ds4, const int32_t* n_dev, int64_t n_ub, const double* T_host,
                      const lw_regmap* reg, float voxel, int32_t reach, float max_d2, float kappa,
                      lw_gn_scratch* gn, double* out64, void* stream);

/* The whole Gauss-Newton loop of odom.py:752-803 on the device, from st->T_pred; result in st->T_reg,
 * st->ok and the stats. One persistent cooperative launch, one grid barrier per iteration. */
int lw_icp_solve(const float* ds4, const int32_t* n_dev, const lw_odom_params* prm, lw_odom_state* st,
                 const lw_regmap* reg, lw_gn_scratch* gn, void* stream);

/* The odometry state (and, with err_dev, the Gauss-Newton error flag) copied to host memory, after everything
 * queued on the stream: the state behind Odometry.stats (odom.py:550-559), in one call. Synchronises the
 * stream. */
int lw_read_state(const lw_odom_state* st_dev, const int32_t* err_dev, lw_odom_state* st_host, int32_t* err_host,
                  void* stream);

/* Deskew and register one frame handed in the caller's device buffers: Odometry._deskew (odom.py:707-709)
 * then Odometry._register (odom.py:752-803, with _downsample :731-737) from T_pred. raw4 [m*4] holds x, y, z,
 * t as measured (16-byte aligned), attr [m]; the points are deskewed to t_mid with twist6 (rho, theta) into
 * fb->f_xyz, thinned into fb->ds_xyz and registered; the result is in st->T_reg, st->ok and the stats
 * (st->n_ds, iters, corr, rms, cond, degen, weak). One launch (the Gauss-Newton kernel deskews and thins the
 * frame before its loop), no host synchronisation. */
int lw_register_frame(const float* raw4, const uint32_t* attr, int64_t m, double t_mid, const float* twist6_host,
                      const double* T_pred_host, const lw_odom_params* prm, lw_odom_state* st, lw_frame_buf* fb,
                      const lw_regmap* reg, lw_gn_scratch* gn, void* stream);

/* lw_register_frame for a frame in the caller's pinned host memory (cudaHostAlloc / cudaHostRegister, mapped for
 * the device), with its result returned there too: the same deskew, thinning and registration (odom.py:707-709,
 * 731-737, 752-803), where the host-side staging of Pipeline.stage (gpu.py:1376-1420) and the state read-back are
 * not separate copies. xyz3 [m*3] (x, y, z), t [m] and attr [m] are read by the launch itself; at its end it
 * writes the state (as lw_read_state would read it) to st_out and the error flag (gn->err) to err_out, also when
 * it gives up. The input buffers must not change and st_out / err_out must not be read until the stream has
 * passed the launch. One launch, no host synchronisation; LW_EINVAL when a buffer is not mapped pinned memory. */
int lw_register_frame_host(const float* xyz3, const float* t, const uint32_t* attr, int64_t m, double t_mid,
                           const float* twist6_host, const double* T_pred_host, const lw_odom_params* prm,
                           lw_odom_state* st, lw_frame_buf* fb, const lw_regmap* reg, lw_gn_scratch* gn,
                           lw_odom_state* st_out, int32_t* err_out, void* stream);

/* ---- integration map (gpu.py:1213-1219) ------------------------------------------------------- */
typedef struct lw_map {
    int64_t* keys;   /* [cap] */
    int32_t* cnt;    /* [cap] hits (keeps counting past LW_MAP_CAP) */
    int64_t* acc;    /* [cap*4] sum of world x, y, z (LW_FIX_W units) and reflectivity over the first LW_MAP_CAP hits */
    float* last;     /* [cap] latest hit time */
    float* first;    /* [cap] earliest hit time (1e30 when empty) */
    int32_t* miss;   /* [cap] carving misses */
    int32_t* bcnt;   /* [cap] scratch, 0 between calls */
    int32_t* lead;   /* [cap] scratch, INT32_MAX between calls */
    int32_t* stats;  /* [2] occupied, dropped */
    int64_t cap;
} lw_map;

/* The filter set of gpu.View (gpu.py:76-98) that the map kernels read. */
typedef struct lw_view {
    float now, persist, min_range, max_range;
    int32_t min_refl, noise_mask, ret_mask, crop_on;
    float crop_lo[3], crop_hi[3];
    float inv_frame_dt;
    int32_t epoch;
    float inv_voxel;
    int32_t map_mask, dyn_on;
    float dyn_settle;
    int32_t carve_on;
    float carve_ratio;
    int32_t carve_min;
    float carve_stale;
} lw_view;

/* Accumulate n points through their frames' poses into the map (gpu.py:373-412). n_dev may be NULL
 * (then n_ub is the count); pslot is [n_ub] scratch. */
int lw_map_insert(const float* xyz, int32_t xyz_stride, const uint32_t* attr, const float* t,
                  const int32_t* frame, const int32_t* n_dev, int64_t n_ub, const float* poses,
                  const lw_view* v, float inv_voxel, lw_map* map, int32_t* pslot, void* stream);

/* Free-space carving of every `every`-th return (gpu.py:469-593). ray_stop is [ceil(n_ub / every)] scratch (the
 * stopping distance of each ray, found from its end point's local plane before the rays are walked). */
int lw_carve(const float* xyz, int32_t xyz_stride, const uint32_t* attr, const int32_t* frame,
             const int32_t* n_dev, int64_t n_ub, const float* poses, int32_t every, float inv_voxel,
             float max_range, int32_t max_steps, lw_map* map, float* ray_stop, void* stream);

/* Classify the map's voxels into the visible set (gpu.py:699-747) and compact it in slot order
 * (gpu.py:1495-1504). Writes count_dev[0]. tiles is [cap/1024 + 1] scratch. */
int lw_map_build(const lw_map* map, const lw_view* v, int32_t min_count, float* out_xyz, uint32_t* out_attr,
                 float* out_t, int32_t* out_dyn, int32_t* tiles, int32_t* count_dev, void* stream);

/* The live ring's visible set (k_classify_live, gpu.py:637-697, with the scan + scatter of Pipeline.build
 * :1466-1504 in live mode), in ring order: every one of the first min(filled, cap) ring slots that is no older
 * than v->persist (when > 0), passes keep_raw, and -- when v->inv_frame_dt > 0 -- whose frame's pose slot holds
 * that frame for v->epoch, deskewed by the frame's twist from its time within the frame; posed by its frame's
 * matrix and inside the crop box. out_* [cap] get the world point, the attribute, the time and, with v->dyn_on,
 * the Motion label from the map's history (settled_near, gpu.py:596-634), else 0. ring_xyz is [cap*3] with
 * cap <= 2^30; tiles is [cap/1024 + 2] scratch; writes count_dev[0]. */
int lw_live_build(const float* ring_xyz, const uint32_t* ring_attr, const float* ring_t, const int32_t* ring_frame,
                  int64_t cap, int64_t filled, const lw_pose_table* pt, const lw_view* v, const lw_map* map,
                  float* out_xyz, uint32_t* out_attr, float* out_t, int32_t* out_dyn, int32_t* tiles,
                  int32_t* count_dev, void* stream);

/* Frame id of each staged point, floor(max(t, 0) * inv_dt), all 0 when inv_dt <= 0 (gpu.py:340-348). */
int lw_frame_ids(const float* t, int64_t n, float inv_dt, int32_t* out, void* stream);

/* Pipeline.stage (gpu.py:1376-1401) in one call: copy a host batch -- xyz_host [n*3], attr_host [n], t_host [n],
 * pinned for an asynchronous copy -- into the device staging buffers and compute its frame ids (frame_dev [n]) with
 * inv_dt as lw_frame_ids does. Three copies and one launch, no host synchronisation. */
int lw_stage_batch(const float* xyz_host, const uint32_t* attr_host, const float* t_host, int64_t n, float* xyz_dev,
                   uint32_t* attr_dev, float* t_dev, float inv_dt, int32_t* frame_dev, void* stream);

/* Buffers of the neighbourhood pass: an open-addressed voxel table of cap (a power of two) slots and the dense
 * per-voxel arrays (at most one voxel per point). */
typedef struct lw_nbr_buf {
    int64_t* keys;       /* [cap] voxel keys, -1 empty (cleared by each call) */
    int64_t* acc;        /* [cap*4] fixed-point sums of x, y, z (LW_FIX_W units) and the point count */
    int32_t* vidx;       /* [cap] dense index of each occupied slot */
    int32_t* v_slot;     /* [cap] slot of each dense voxel */
    int32_t* slot_of_pt; /* [pt_cap] voxel slot of each point, -1 when the table was full */
    float* v_xyz;        /* [cap*3] voxel centroids, in slot order */
    int32_t* v_w;        /* [cap] points per voxel */
    float* v_cnt;        /* [cap] point-weighted neighbour count */
    float* v_nrm;        /* [cap*3] unit normals */
    float* v_curv;       /* [cap] curvature */
    int32_t* tiles;      /* [cap/1024 + 1] scan scratch */
    int32_t* m;          /* [1] voxels */
    int64_t cap, pt_cap;
} lw_nbr_buf;

/* Neighbourhoods of the first n points (gpu.py:777-905, Pipeline.neighborhoods :1531-1557): the points are summed
 * into voxels radius / 3 wide; each voxel's neighbours are the voxels whose centroid lies within `radius`
 * (0 < radius <= 4 m) of its own, and their point-weighted count, the normal of their covariance's smallest
 * eigenvalue turned toward `sensor` (host float[3]) and the curvature (smallest eigenvalue / trace) are handed to
 * every point of the voxel: out_cnt [n] int32 (rounded), with want_normals out_nrm [n*3] and out_curv [n]. Sums
 * are exact fixed point and float64, so each point's answers do not depend on thread order. A point whose voxel
 * did not fit in the table gets count 2^30, normal (0, 0, 1), curvature 0. */
int lw_neighborhoods(const float* xyz, int32_t xyz_stride, const int32_t* n_dev, int64_t n_ub, float radius,
                     int32_t want_normals, const float* sensor, lw_nbr_buf* nb, int32_t* out_cnt, float* out_nrm,
                     float* out_curv, void* stream);

/* Prior-map voxel table (prior_map.py:57-123, voxel_downsample :169-203): cap slots (a power of two, at most
 * 2^30) filled chunk by chunk. Clear keys to -1 (0xFF bytes), acc and stats to 0 and first to 0x7F bytes before the
 * first chunk (lw_vox_clear does it). */
typedef struct lw_vox_buf {
    int64_t* keys;       /* [cap] voxel keys of floor(p / voxel) (gpu.py voxel_key_ijk), -1 empty */
    int64_t* acc;        /* [cap*8] per voxel: x, y, z offsets from the voxel centre (units of
                          * lw_vox_offset_units(voxel) per metre), r, g, b, intensity (LW_VOX_FIX_ATTR units), points */
    int64_t* first;      /* [cap] lowest point index that reached the voxel */
    int32_t* order;      /* [cap] slot of the j-th voxel; voxels are numbered in the order of their first point */
    int32_t* slot_of_pt; /* [pt_cap] scratch: slot of each point of a chunk, -1 when the probe window was full */
    int32_t* tiles;      /* [pt_cap/1024 + 1] scratch */
    int64_t* stats;      /* [2] voxels so far, points dropped (probe window full) */
    int64_t cap, pt_cap;
} lw_vox_buf;

#define LW_VOX_FIX_ATTR 65536.0 /* prior-map voxel table: units per unit of colour and intensity, 2^16 */

/* Units per metre of a prior-map voxel's offset sums: 2^(30 - e) for the smallest e with voxel < 2^e, so a point's
 * offset from its voxel centre is below 2^29 units. */
double lw_vox_offset_units(float voxel);

/* Reset the voxel table for a new cloud. */
int lw_vox_clear(lw_vox_buf* vb, void* stream);

/* Add n points (n <= pt_cap <= 2^30) to their voxels (k_vox_insert, prior_map.py:57-91), voxel in [1e-6, 1e6] m:
 * xyz [n*xyz_stride] (stride 3 or 4, finite), intensity [n] and rgb [n*3] optional (NULL sums zeros). index0
 * is the number of points of the cloud inserted by earlier calls, so that every point has its own index; the
 * voxels first reached by this chunk are appended to `order` in the order of their first point. A point whose
 * 128-slot probe window is full counts in stats[1] and is left out (the reference raises on it). */
int lw_vox_insert(lw_vox_buf* vb, const float* xyz, int32_t xyz_stride, const float* intensity, const float* rgb,
                  int64_t n, int64_t index0, float voxel, void* stream);

/* The first min(stats[0], m_cap) voxels as dense arrays (k_vox_emit, prior_map.py:100-123): out_xyz [m*3] the
 * mean position (voxel centre + mean offset), out_rgb [m*3] and out_intensity [m] the mean colour and intensity,
 * out_cnt [m] the point count; every output may be NULL. */
int lw_vox_emit(const lw_vox_buf* vb, float voxel, int64_t m_cap, float* out_xyz, float* out_rgb,
                float* out_intensity, int32_t* out_cnt, void* stream);

/* Buffers of the normal estimation: a table of cells slightly wider than the radius (cap, a power of two, at
 * least twice the points, at most 2^30) and the points grouped by cell. */
typedef struct lw_pca_buf {
    int64_t* keys;       /* [cap] cell keys, -1 empty (cleared by each call) */
    int32_t* cell_cnt;   /* [cap] points per cell */
    int32_t* cell_start; /* [cap] first position of each cell's points in `sorted` */
    int32_t* slot_of_pt; /* [pt_cap] cell slot of each point, -1 when the probe window was full */
    int32_t* rank_of_pt; /* [pt_cap] position of each point within its cell */
    float* sorted;       /* [pt_cap*4] the points grouped by cell: x, y, z and the point index (int32 bits) */
    int32_t* tiles;      /* [cap/1024 + 1] scan scratch */
    int32_t* stats;      /* [2] points placed, points dropped */
    int64_t cap, pt_cap;
} lw_pca_buf;

/* PCA normal and planarity of each of n points (n <= pt_cap <= 2^30) from all points within `radius` (1e-4 to 16 m,
 * |q - p|^2 <= radius^2 in float32) (k_normals, prior_map.py:126-166, normals :206-219): out_nrm [n*3] the unit
 * eigenvector of the covariance's smallest eigenvalue, out_planarity [n] (l_mid - l_min) / max(l_max, 1e-12);
 * both zero for a point with fewer than 4 neighbours (itself included) or one the table could not place. The
 * neighbour offsets and their products are summed in int64 fixed point (2^20 and 2^40 units of the radius' power
 * of two), the covariance and its eigen-decomposition are float64: the answers do not depend on thread order.
 * Exact up to 2^23 neighbours per point. */
int lw_normals(const float* xyz, int32_t xyz_stride, int64_t n, float radius, lw_pca_buf* pb, float* out_nrm,
               float* out_planarity, void* stream);

/* LVXR recordings (host). lw_lvxr_decode decodes a whole recording held in memory into every firing with its
 * exact time, the empty ones included (lvxr.py read_firings :189-260, the datagrams of record.rs / point.rs):
 * n firings of up to R returns each, time-ordered. lw_lvxr_info reports n, R, the device type, the profile and the
 * firing interval (s); lw_lvxr_copy fills t [n] float64 s, xyz [n*R*3] float32 m (sensor frame, zero where a return
 * slot is empty), refl / tag / valid [n*R] uint8 and direction [n*3] float32 (NaN where the data gives none); the
 * decoded recording is host memory owned by the handle until lw_lvxr_free. */
typedef struct lw_lvxr lw_lvxr;
int lw_lvxr_decode(const uint8_t* data, int64_t size, lw_lvxr** out);
int lw_lvxr_info(const lw_lvxr* r, int64_t* n_firings, int32_t* returns, int32_t* dev_type, int32_t* profile,
                 double* interval_s);
int lw_lvxr_copy(const lw_lvxr* r, double* t, float* xyz, uint8_t* refl, uint8_t* tag, uint8_t* valid,
                 float* direction);
void lw_lvxr_free(lw_lvxr* r);

/* Clear the integration map (gpu.py:1305-1313). */
int lw_map_clear(lw_map* map, void* stream);

/* ---- perception (perception.py) -------------------------------------------------------------- */

/* Ground labels of n points (perception.py:29-111, Perception.ground :458-483): grid minimum per toroidal
 * 2048 x 2048 cell, support within `thick`, the lowest supported minimum of the 5 x 5 cells around a point plus
 * slope_step per cell of Chebyshev distance, ground when within `thresh`; hag = height above that ground.
 * cell_min [2048*2048] (1e30) and cell_sup [2048*2048] (0) must hold their cleared values between calls; the call
 * restores the cells it touched. nrm [n*3] is read only with use_normals. */
int lw_ground(const float* xyz, int32_t xyz_stride, const float* nrm, const int32_t* n_dev, int64_t n_ub, float cell,
              float thick, int32_t min_sup, float thresh, float slope_step, int32_t use_normals, float nz_min,
              float* cell_min, int32_t* cell_sup, int32_t* out_gnd, float* out_hag, void* stream);

/* Buffers of the Euclidean clustering; "between calls" values are restored by every call. */
typedef struct lw_cluster_buf {
    int64_t* keys;       /* [cap] voxel keys, -1 between calls */
    int64_t* acc;        /* [cap*4] fixed-point x, y, z sums (LW_FIX_W) and point count, 0 between calls */
    int32_t* first;      /* [cap] lowest point index per voxel, INT32_MAX between calls */
    int32_t* vidx;       /* [cap] node of a slot */
    int32_t* slot_of_pt; /* [pt_cap] */
    int32_t* tiles;      /* [pt_cap/1024 + 2] */
    int32_t* node_slot;  /* [pt_cap] slot of a node */
    float* v_xyz;        /* [pt_cap*3] node centroids */
    int32_t* v_w;        /* [pt_cap] node point counts */
    int32_t* edge_off;   /* [pt_cap + 1] */
    int32_t* edges;      /* [edge_cap] neighbour lists */
    int32_t* label;      /* [pt_cap] component of a node: its smallest node index */
    int64_t* st_sum;     /* [pt_cap*4] per-root fixed-point sums and count, 0 between calls */
    float* st_lo;        /* [pt_cap*3] per-root minimum corner, +1e30 between calls */
    float* st_hi;        /* [pt_cap*3] per-root maximum corner, -1e30 between calls */
    int32_t* dense;      /* [pt_cap] dense cluster id of a root, -1 */
    float* out_cnt;      /* [max_out] points per cluster */
    float* out_cen;      /* [max_out*3] centroids */
    float* out_lo;       /* [max_out*3] */
    float* out_hi;       /* [max_out*3] */
    int32_t* m;          /* [1] nodes of the last call */
    int32_t* n_clusters; /* [2] clusters kept, clusters before the max_out cap */
    int32_t* err;        /* [1] non-zero when a buffer was too small or a bounded loop gave up */
    int64_t cap, pt_cap, edge_cap;
} lw_cluster_buf;

/* Connected components of the (non-ground) points' voxels (perception.py:114-271, Perception.cluster :487-567):
 * voxels of size `voxel` linked when their centroids are within `connect`; clusters with >= min_pts points get
 * dense ids 0.. in node order (a node's order is its first point's), at most max_out; out_cid [n] per point. */
int lw_cluster(const float* xyz, int32_t xyz_stride, const int32_t* gnd, int32_t use_ground, const int32_t* n_dev,
               int64_t n_ub, float voxel, float connect, float min_pts, int32_t max_out, lw_cluster_buf* cb,
               int32_t* out_cid, void* stream);

/* ---- prior-map grid and batched localisation ICP (mapgrid.py, localize.py) -------------------------- */

/* A dense grid over a prior map (mapgrid.py:1-33, 207-296): the n map points sorted by cell (start[c] ..
 * start[c+1] are cell c's points), a jump-flooded nearest point per cell and a byte distance field in cm. A map
 * point is one 16-byte record (x, y, z, planarity), so the nearest-point scans gather one aligned vector each. */
typedef struct lw_prior_grid {
    float* xyz;       /* [n*4] map points sorted by cell: x, y, z, planarity (16-byte aligned) */
    float* nrm;       /* [n*3] unit normals */
    int32_t* start;   /* [ncell+1] */
    int32_t* nn;      /* [ncell] flooded nearest point or -1 */
    uint8_t* df;      /* [ncell] distance to it in cm, 255 beyond the band */
    uint64_t* seed;   /* [ncell] build scratch */
    int32_t* nn2;     /* [ncell] build scratch */
    float origin[3];
    float cell, inv_cell;
    int32_t nx, ny, nz, pad_;
    int64_t n, ncell;
} lw_prior_grid;

/* Build nn and df from the sorted points (k_seed, k_unpack, k_jfa x (8, 4, 2, 1, 1), k_df: mapgrid.py:105-170,
 * 272-296). Seeds are 64-bit (no 2^23-point limit) and the flood is double buffered (deterministic). */
int lw_prior_grid_build(lw_prior_grid* g, void* stream);

/* Distance of n points (pts [n*3]) posed by T (row-major 4x4, host) to the nearest map point, 1e3 beyond the
 * band (mapgrid.py:173-194, PriorGrid.distances :298-305). */
int lw_prior_distances(const lw_prior_grid* g, const float* pts, int64_t n, const double* T_host, float* out,
                       void* stream);

/* Coarse search scores (localize.py:55-96, k_score_grid): for every position pos[i] (float xyz, i < n_pos) and
 * heading yaw0 + j dyaw (j < n_yaw <= LW_SCORE_MAX_YAW), the soft count of the n_pts scan points pts [n_pts*3]
 * (gravity-aligned sensor frame) near the map: the sum over points whose cell distance d (cm, the grid's df) is
 * below tau_cm of 1 - d^2 / tau_cm^2, formed exactly from integer sums (the reference adds float32 terms in point
 * order). out[i*n_yaw + j]; -1 where the position lies outside the grid or within free_cm of a mapped surface.
 * Needs the built grid (df); a buffer may be null when its count is 0. pos_stride (>= 1) only sets the thread layout: when positions i and i + pos_stride
 * are neighbours along x (ny for a meshgrid with y inner, as localize.py:428-432 builds), a warp's gathers share
 * cache lines; 1 for any list. */
#define LW_SCORE_MAX_YAW 1024
int lw_score_grid(const lw_prior_grid* g, const float* pts, int32_t n_pts, const float* pos, int64_t n_pos,
                  int64_t pos_stride, int32_t n_yaw, float yaw0, float dyaw, float tau_cm, float free_cm, float* out,
                  void* stream);

/* The same soft count for a list of hypotheses hyp [n_hyp*4] = (x, y, z, yaw), 16-byte aligned
 * (localize.py:99-123, k_score_list). */
int lw_score_list(const lw_prior_grid* g, const float* pts, int32_t n_pts, const float* hyp, int64_t n_hyp,
                  float tau_cm, float* out, void* stream);

/* Local maxima of lw_score_grid's scores laid out as (nz heights, nx, ny, n_yaw) -- the meshgrid order of
 * localize.py:428-432 -- by the rule of localize.py:450-483 (_local_maxima): a positive score, at least
 * min_score, no less than any of the 26 (x, y, heading) neighbours at the same height (x / y neighbours outside
 * the grid skipped, headings wrapping). Appends up to cap survivors as (idx [cap] int64, val [cap]) in no
 * particular order; count_dev[0] = the number of survivors (may exceed cap). Clears count_dev on the stream. */
int lw_score_maxima(const float* scores, int32_t nz, int32_t nx, int32_t ny, int32_t n_yaw, float min_score,
                    int32_t cap, int64_t* idx, float* val, int32_t* count_dev, void* stream);

/* The headings' float32 cosines and sines lw_score_grid poses points with: yaw_j = yaw0 + j dyaw in float32
 * (localize.py:82), its cosine and sine in float64 rounded to float32. Host only; c and s hold n_yaw floats. */
void lw_score_yaw_table(int32_t n_yaw, float yaw0, float dyaw, float* c, float* s);

/* Buffers of the batched ICP: every hypothesis has its own range of points (tile_lo .. scan_end; hypotheses may
 * share one scan) and pose (T, in and out). The points are cut into tiles of at most `tile` points that never
 * span two hypotheses: hypothesis h owns tiles hyp_tile[h] .. hyp_tile[h+1]. */
typedef struct lw_loc_batch {
    float* pts;         /* [pts_cap*4] x, y, z, unused */
    int32_t* scan_end;  /* [n_hyp] end (exclusive) of each hypothesis' points */
    int32_t* tile_hyp;  /* [n_tiles] hypothesis of each tile */
    int32_t* tile_lo;   /* [n_tiles] first point of each tile */
    int32_t* hyp_tile;  /* [n_hyp+1] first tile of each hypothesis */
    double* T;          /* [n_hyp*16] row-major poses, updated in place */
    double* tile_part;  /* [n_tiles*32] float64 tile partials (scratch) */
    int32_t* moved;     /* [moved_cap] largest step of each iteration (scratch) */
    int32_t* next;      /* [moved_cap + 1] tile counters of the iterations and the evaluation (scratch) */
    int32_t* count;     /* [n_hyp] matched points in the last iteration */
    int32_t* eval;      /* [n_hyp*3] points within 3 / 5 / 10 cm of the map at the final pose */
    uint32_t* bar;      /* [2] grid barrier, zero before the first use */
    int32_t* err;       /* [1] set when a bounded wait gave up */
    int32_t* iters_run; /* [1] iterations run over all stages */
    int32_t* dims;      /* [2] n_hyp, n_tiles read on the device (a graph replayed over changing batches), or NULL */
    int64_t pts_cap;    /* points the pts buffer holds; tiles and scan ends are clamped to it */
    int32_t moved_cap, grid_cap;
} lw_loc_batch;

/* Point-to-plane ICP of every hypothesis at once against the grid (k_icp_batch / k_reduce_batch / the host
 * solve of GlobalLocalizer._icp, localize.py:126-179, 517-553, then k_eval_batch :182-205), in one cooperative
 * launch: stages k = 0..n_stages-1 of iters[k] iterations with correspondence distance dmax[k] (max_d2 and the
 * Geman-McClure c2 = (dmax/2)^2 are formed in double and rounded to float, as the reference's host does); a
 * hypothesis with fewer than min_count matches keeps its pose; a stage ends when no hypothesis moved 2e-4
 * (n_stages = 0 only evaluates). With b->dims set, n_hyp and n_tiles are capacities and the counts are read on
 * the device. tile: points per tile (a multiple of 32 up to 2048), each tile worked by one warp; the host's tiling
 * must use the same value. blocks_per_sm: the register budget, 2 to 6 resident 256-thread CTAs per SM (0 = 3).
 * grid <= 0 picks one full wave. */
int lw_loc_icp_batch(const lw_prior_grid* g, lw_loc_batch* b, int32_t n_hyp, int32_t n_tiles, int32_t tile,
                     int32_t n_stages, const double* dmax, const int32_t* iters, float alpha, int32_t min_count,
                     int32_t blocks_per_sm, int32_t grid, void* stream);

/* ---- learned initial pose (no counterpart in the reference: its odometry predicts with constant velocity) ---- */

/* A point-set network proposing the ICP start pose: a shared per-point MLP 3 -> 64 -> 128 -> 256 (ReLU), a max
 * over the LW_NET_P points of each set, the frame's and the map patch's codes concatenated (512), then
 * 512 -> 128 (ReLU) -> 6: an se(3) step (tx, ty, tz, rx, ry, rz) in the predicted sensor frame, so that
 * T = T_pred * exp(step). Weights and activations are bf16 with float32 accumulation; layers 2 and 3 run on the
 * tensor cores (tcgen05.mma, accumulators in TMEM). Parameters live in one flat float32 master buffer (Adam)
 * with a bf16 copy the kernels read, at the LW_NET_OFF_* element offsets. */
#define LW_NET_P 1024
#define LW_NET_OFF_W1 0        /* [64][3]   */
#define LW_NET_OFF_B1 192      /* [64]      */
#define LW_NET_OFF_W2 256      /* [128][64] */
#define LW_NET_OFF_B2 8448     /* [128]     */
#define LW_NET_OFF_W3 8576     /* [256][128] */
#define LW_NET_OFF_B3 41344    /* [256]     */
#define LW_NET_OFF_WH1 41600   /* [128][512] */
#define LW_NET_OFF_BH1 107136  /* [128]     */
#define LW_NET_OFF_WH2 107264  /* [6][128]  */
#define LW_NET_OFF_BH2 108032  /* [6]       */
#define LW_NET_NPARAM 108040   /* padded to a multiple of 8 */

typedef struct lw_initnet {
    float* master;    /* [LW_NET_NPARAM] float32 weights (what Adam updates) */
    uint16_t* w;      /* [LW_NET_NPARAM] bf16 copy the kernels read (16-byte aligned) */
    float* grad;      /* [LW_NET_NPARAM] gradient of the last backward pass */
    float* adam_m;    /* [LW_NET_NPARAM] */
    float* adam_v;    /* [LW_NET_NPARAM] */
    float* out_scale; /* [6] output scale: step = network output * out_scale */
    float in_scale;   /* input points are multiplied by this (1 / metres) */
    int32_t pad_;
} lw_initnet;

/* Forward pass of n samples: sets [2n][LW_NET_P][4] (x, y, z, unused; set 2s is sample s's frame, 2s+1 its map
 * patch, both in the predicted sensor frame). Writes pooled [2n][256] (the max of each channel), argmax [2n][256]
 * (the first point attaining it), hid [n][128] (the head's hidden layer, bf16 values) and step [n][6]
 * (out_scale applied). err [1] is set when a bounded wait gave up. */
int lw_net_forward(const lw_initnet* net, const float* sets, int32_t n, float* pooled, int32_t* argmax, float* hid,
                   float* step, int32_t* err, void* stream);

/* Scratch of the backward pass for up to n_cap samples (sizes in floats unless stated). */
typedef struct lw_net_scratch {
    float* dz3;       /* [2n*256] */
    uint16_t* h2g;    /* [2n*256*128] bf16: layer-2 activations of each channel's argmax point */
    float* d2t;       /* [128][2n*256] */
    float* h1t;       /* [65][2n*256]: layer-1 activations, then a row of ones */
    float* d1t;       /* [64][2n*256] */
    float* xt;        /* [4][2n*256]: the scaled inputs, then a row of ones */
    float* dzh;       /* [n][128] */
    float* dout;      /* [n][6] */
    float* dpool;     /* [2n][256] */
    float* part;      /* [64 * 8448] split-K partials */
    float* loss;      /* [n] per-sample loss */
    int32_t n_cap;
    int32_t pad_;
} lw_net_scratch;

/* Loss sum_s sum_j w[j] * (out[s][j] - target[s][j] / out_scale[j])^2 / n and its gradient with respect to the
 * bf16 weights, into net->grad (backpropagation through the max: only each channel's argmax point receives
 * gradient). target [n][6] is the true step. Per-sample losses in scr->loss. */
int lw_net_backward(const lw_initnet* net, const float* sets, int32_t n, const float* pooled, const int32_t* argmax,
                    const float* hid, const float* step, const float* target, const float* w_loss,
                    lw_net_scratch* scr, void* stream);

/* One Adam step (t >= 1) on the master weights with decoupled weight decay, then the bf16 copy. */
int lw_net_adam(lw_initnet* net, int32_t t, float lr, float beta1, float beta2, float eps, float weight_decay,
                void* stream);

/* Deterministic initialisation (He-uniform weights from `seed`, zero biases and moments, out_scale untouched). */
int lw_net_init(lw_initnet* net, uint64_t seed, void* stream);

/* The two point sets of the current frame, in the frame of pose T (row-major 4x4 float64 on the device, e.g. the
 * state's T_pred). Frame set: LW_NET_P points taken at an even stride from the thinned frame (ds_xyz, n_ds on the
 * device). Map set, with voxel > 0 (the registration voxel): for each frame-set point, the nearest registration
 * voxel mean among the 27 voxels around it at T (the point itself where none is occupied); with voxel <= 0: the
 * registration voxel means within `radius` of T's origin, in slot order at an even stride (cand [reg cap] and
 * tiles [reg cap / 1024 + 2] are then scratch). sets_out [2][LW_NET_P][4]; count [2] receives the frame's point
 * count and the patch's candidate count. */
int lw_net_sets(const float* ds_xyz, const int32_t* n_ds, const lw_regmap* reg, const double* T, float radius,
                float voxel, float* sets_out, int32_t* cand, int32_t* tiles, int32_t* count, void* stream);

/* lw_odom_finalize with the learned start pose: after the frame is deskewed and thinned with the predicted
 * motion, the network sees the frame and the map patch around the constant-velocity prediction T_pred and the
 * registration starts from (and its prior is anchored at) T_pred * exp(step) instead. work: sets [2*LW_NET_P*4],
 * pooled [512], argmax [512] (int), hid [128], step [6], err [1] (int) floats, cand / tiles as lw_net_sets. */
typedef struct lw_net_work {
    float* sets;
    float* pooled;
    int32_t* argmax;
    float* hid;
    float* step;
    int32_t* err;
    int32_t* cand;
    int32_t* tiles;
    int32_t* count;
    float radius; /* map patch radius when voxel <= 0 */
    float voxel;  /* > 0: the map set is the nearest registration voxel mean of each frame-set point */
} lw_net_work;

int lw_odom_finalize_net(int32_t k, int64_t m_ub, const lw_odom_params* prm, lw_odom_state* st, lw_frame_buf* fb,
                         lw_regmap* reg, lw_gn_scratch* gn, lw_pose_table* pt, int32_t epoch, lw_traj_rec* traj,
                         int64_t traj_cap, const lw_initnet* net, lw_net_work* work, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LIVOX_B200_H */
