/*
 * mrpnn_b200.h - C ABI of the B200-native MRPNN cloud renderer.
 *
 * Plain pointers, sizes and POD structs only. Every entry point returns an
 * int status (mr_status); mr_last_error() gives the message of the last
 * failure on the calling thread. Device pointers are CUDA device memory on
 * the current device; `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the reference project).
 */
#ifndef MRPNN_B200_H
#define MRPNN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float x, y, z; } mr_float3;

typedef enum {
  MR_OK = 0,
  MR_ERR_ARG = 1,         /* invalid argument (size, pointer, range) */
  MR_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  MR_ERR_TIMEOUT = 3,     /* mr_sync / mr_render_host_wait watchdog expired */
  MR_ERR_LOOP_CAP = 4,    /* a device loop hit its iteration cap and reported it */
  MR_ERR_STATE = 5,       /* call made in the wrong state (e.g. render before update) */
  MR_ERR_NOMEM = 6,       /* device allocation failed */
  MR_ERR_UNSUPPORTED = 7  /* feature not built into this library */
} mr_status;

/* core/volume.hpp:88-90 VolumeRender::RenderType (RPNN's weights are not in
 * the reference tree and it is not supported here), plus the marching form of
 * the neural render, NNPredict<Type::marching_MRPNN> (core/render.cuh:524-633):
 * the camera ray is marched in 1/1023 steps of its box length (negative
 * densities skip that distance), the network's point is drawn among the
 * marched samples in proportion to their absorbed share, and with a surface
 * IOR (mr_volume_set_surface_ior) the first medium sample is a dielectric
 * surface that reflects or refracts the ray. */
typedef enum { MR_RT_PT = 0, MR_RT_RPNN = 1, MR_RT_MRPNN = 2, MR_RT_MARCHING_MRPNN = 3 } mr_render_type;

/* Arithmetic of the radiance-predictor MLP.
 * FP32: CUDA cores, the reference's arithmetic order.
 * BF16: tcgen05 tensor cores, BF16 operands, FP32 accumulation.
 * FP8:  tcgen05 tensor cores, E4M3 operands with a power-of-two scale per
 *       layer (weights) and per row (activations), FP32 accumulation. */
typedef enum { MR_PREC_FP32 = 0, MR_PREC_BF16 = 1, MR_PREC_FP8 = 2 } mr_precision;

/* What mr_volume_read copies back. */
typedef enum {
  MR_READ_DENSITY = 0,   /* res^3, x-major */
  MR_READ_MIP = 1,       /* level k: (256>>k)^3 */
  MR_READ_VARIANCE = 2,  /* level k: (256>>k)^3 */
  MR_READ_TR = 3,        /* level k: (128>>k)^3 */
  MR_READ_HGLUT = 4      /* 512 x 512, index i + j*512 (i: cos bin, j: cone-angle bin) */
} mr_read_what;

typedef struct mr_volume mr_volume;
typedef struct mr_network mr_network;

/* One render request. Mirrors the arguments of VolumeRender::Render
 * (core/volume.hpp:141) plus the device-side settings the reference keeps in
 * __device__ globals (core/render.cuh:9-17): scatter_rate, tr_scale,
 * enviroment_exp. */
typedef struct {
  int32_t width, height;
  mr_float3 ori;          /* camera position; forward = normalize(-ori) */
  mr_float3 up, right;    /* screen half-extent vectors (tan(fov/2) scaled) */
  mr_float3 light_dir;    /* direction towards the light (normalised inside) */
  mr_float3 light_color;
  float alpha;            /* extinction scale */
  float g;                /* Henyey-Greenstein asymmetry */
  mr_float3 scatter_rate; /* per-channel albedo (SetScatterRate) */
  float tr_scale;         /* NEE step scale (SetTrScale), normally 1 */
  mr_float3 env_color;    /* radiance of escaped rays (constant environment), 0 = black; with an
                             environment map (mr_volume_set_hdri) the map's scale (SetEnvExp) */
  int32_t max_bounces;    /* multiScatter */
  int32_t spp;            /* samples per pixel (PT); neural renders 1 primary sample per pass */
  uint32_t seed;          /* Philox key */
  uint32_t sample_offset; /* index of the first sample (progressive accumulation) */
  int32_t render_type;    /* mr_render_type */
  int32_t precision;      /* mr_precision (MRPNN only) */
  int32_t sampler;        /* mr_sampler for the descriptor gather (MRPNN only) */
} mr_render_params;

/* How the neural gather samples the mip / transmittance / HG tables.
 * EXACT: fp32 trilinear in software (bit-stable, the oracle's arithmetic).
 * TEXTURE: the texture units' trilinear filter for the mip and transmittance
 * tables, as the reference samples its texture references
 * (core/volume.cu:1289-1298): 8-bit interpolation weights, several times fewer
 * instructions per sample; the HG table keeps the fp32 bilinear filter (its
 * lookups go through the load path, off the busy texture path). */
typedef enum { MR_SAMPLER_EXACT = 0, MR_SAMPLER_TEXTURE = 1 } mr_sampler;

/* Library version string. */
const char* mr_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char* mr_last_error(void);

/* ---- volume (replaces VolumeRender: core/volume.hpp:45-146) ---------------- */

/* VolumeRender(int resolution) + MallocMemory (core/volume.cu:748-773,831-833). */
int mr_volume_create(int32_t resolution, mr_volume** out);
/* VolumeRender(string path) (core/volume.cu:835-911): reads <path>.bin if it
 * exists (int32 resolution r, then r^3 fp32, index (x*r+y)*r+z), else a .txt
 * file (r, then r^3 whitespace-separated values) or a .vox file (256^3;
 * header lines start with 'w', 'h' or 'd'; data lines hold 64 integers, each
 * value * 64 / 255), then creates the volume and runs mr_volume_update. After
 * reading a .txt or .vox file it writes <path>.bin as the reference does,
 * unless write_cache is 0. A missing or malformed file is MR_ERR_ARG (the
 * reference printed "File not found!" and returned). */
int mr_volume_load(const char* path, int32_t write_cache, mr_volume** out, void* stream);
/* The parsing step of mr_volume_load alone (host only, no device use):
 * *resolution receives r; host_out (may be NULL to query r) receives r^3
 * floats if capacity allows. */
int mr_volume_file_read(const char* path, float* host_out, size_t capacity, int32_t* resolution);
/* ~VolumeRender (core/volume.cu:913-936). */
int mr_volume_destroy(mr_volume* v);
/* SetDatas / SetData (core/volume.cu:938-944): host array, index (x*res+y)*res+z. */
int mr_volume_set_data(mr_volume* v, const float* host_data, size_t count);
/* Same, from device memory, stream-ordered. */
int mr_volume_set_data_device(mr_volume* v, const float* dev_data, size_t count, void* stream);
/* Update() (core/volume.cu:1203-1316): global majorant, density mip pyramid
 * 256^3..1^3 and its 2x2x2 variance pyramid. */
int mr_volume_update(mr_volume* v, void* stream);
/* Update_TR(lightDir, alpha) (core/volume.cu:1346-1424): light-transmittance
 * pyramid 128^3..1^3. Skipped when light and alpha are unchanged. */
int mr_volume_update_tr(mr_volume* v, mr_float3 light_dir, float alpha, void* stream);
/* UpdateHGLut(g) (core/volume.cu:1161-1183): 512x512 cone-averaged HG table.
 * Skipped when g and seed are unchanged. */
int mr_volume_update_hglut(mr_volume* v, float g, uint32_t seed, void* stream);
/* SetHDRI (core/volume.cu:1426-1458) from pixels: host_rgba is w x h RGBA
 * fp32, row 0 looking straight up; direction d maps to column
 * u = atan2(-d.z, d.x) / 2pi + 1/2 and row v = acos(d.y) / pi, sampled
 * bilinearly with wrap (SkyBox, core/render.cuh:57-61). Escaped rays of every
 * render of this volume then see map(d) * env_color (env_color plays the part
 * of SetEnvExp); neural renders also draw each pass's light from the map or
 * from the directional light as the reference's Render does
 * (core/volume.cu:417-432; see mr_render). Waits for the device when it
 * replaces a map. */
int mr_volume_set_hdri(mr_volume* v, const float* host_rgba, int32_t w, int32_t h);
/* SetHDRI(path): a Radiance RGBE (.hdr) file (core/hdr_loader.h:249). */
int mr_volume_load_hdri(mr_volume* v, const char* path);
/* Removes the map: escaped rays see the constant env_color again. */
int mr_volume_clear_hdri(mr_volume* v);
/* load_hdr_float4 (core/hdr_loader.h:249) alone, host only: *width, *height
 * receive the size; host_rgba (may be NULL to query the size) receives
 * width*height RGBA floats (alpha 0) if capacity allows. */
int mr_hdr_read(const char* path, float* host_rgba, size_t capacity, int32_t* width, int32_t* height);
/* SetSurfaceIOR (core/volume.cu:1490-1493): index of refraction of the
 * surface of MR_RT_MARCHING_MRPNN renders; <= 0 (the default -1) = no surface. */
int mr_volume_set_surface_ior(mr_volume* v, float ior);
/* VolumeRender::max_density after mr_volume_update. */
int mr_volume_max_density(const mr_volume* v, float* out);
int mr_volume_resolution(const mr_volume* v, int32_t* out);
/* Copy one level of a volume-side table back to the host (synchronous). */
int mr_volume_read(const mr_volume* v, int32_t what, int32_t level, float* host_out, size_t count);

/* ---- network (replaces the NNWeight.cuh constants: core/NNWeight.cuh) ------ */

/* Upload MR_WEIGHT_TOTAL fp32 weights in the blob layout of mrpnn_weights.h.
 * `stencil_xyz` is 160 x 3 floats of stencil directions; NULL selects the
 * reference's own directions (core/vector.cu:77-172), the ones the weights
 * of core/NNWeight.cuh were trained on. */
int mr_network_create(const float* host_weights, size_t count, const float* stencil_xyz,
                      mr_network** out);
int mr_network_destroy(mr_network* net);

/* The default 160-point stencil (used when mr_network_create gets NULL): the
 * reference's directions, core/vector.cu:77-172 (Spn0..Spn4, SpVn5..SpVn7),
 * as SphereRandom3 reads them with the identity frame: 480 floats. */
int mr_builtin_stencil(float* host_out, size_t count);
/* An alternative stencil in the same shell layout (no reference
 * counterpart): golden-angle spirals, for networks trained on it. 480 floats. */
int mr_spiral_stencil(float* host_out, size_t count);
/* Xavier-uniform initial weights for the blob layout (zero biases), from
 * Philox with the given seed: MR_WEIGHT_TOTAL floats. */
int mr_weights_xavier(uint32_t seed, float* host_out, size_t count);

/* ---- rendering ------------------------------------------------------------- */

/* VolumeRender::Render(int2 size, ...) (core/volume.cu:410-467) into caller
 * device memory: dev_rgb = width*height*3 fp32, row-major, mean radiance over
 * the samples. PT = delta tracking; MRPNN = neural form (network required;
 * call mr_volume_update_tr / _hglut first or let the call do it). With an
 * environment map on the volume, each MRPNN pass (sample_offset) takes its
 * light from the map with probability 4e / (4e + max(light_color)),
 * e = max(env_color): direction = the R2 point sample_offset on the sphere,
 * colour = map * env_color * 4 / that probability, else the directional
 * light with colour / (1 - probability); the transmittance pyramid is rebuilt
 * for the chosen light. The coin is Philox(seed; sample_offset, 0, 0, 7). */
int mr_render(mr_volume* v, const mr_network* net, const mr_render_params* p, float* dev_rgb,
              void* stream);
/* Same, synchronous, into host memory (the reference returns vector<float3>). */
int mr_render_host(mr_volume* v, const mr_network* net, const mr_render_params* p, float* host_rgb);
/* Pipelined form of mr_render_host for a stream of frames (VolumeRender::Render,
 * core/volume.cu:410-467, called once per frame): renders on `stream` into one
 * of two device frames owned by the volume, used in turn, and copies the frame
 * to host_rgb on a copy stream owned by the volume, so that the copy of one
 * frame overlaps the render of the next. Returns once both are queued;
 * *ticket (may be NULL) numbers the frame for mr_render_host_wait. host_rgb
 * must stay valid until that wait; page-locked memory lets the copy overlap. */
int mr_render_host_async(mr_volume* v, const mr_network* net, const mr_render_params* p, float* host_rgb,
                         void* stream, int64_t* ticket);
/* Blocks until frame `ticket` (and every frame issued before it) is in host
 * memory; ticket < 0 waits for all frames. timeout_ms < 0 waits without limit;
 * MR_ERR_TIMEOUT when the copy is still running after timeout_ms. */
int mr_render_host_wait(mr_volume* v, int64_t ticket, int32_t timeout_ms);
/* Delta tracking with FP64 accumulation: adds this call's per-pixel radiance
 * sums and sums of squares (width*height*3 doubles each, caller-zeroed) so
 * that many calls build a high-spp reference image. */
int mr_render_accumulate_f64(mr_volume* v, const mr_render_params* p, double* dev_sum,
                             double* dev_sumsq, void* stream);

/* RadiancePredict network body (core/radiancePredict.cu:370-485) on n
 * descriptors: dev_desc = n x 576 fp32 ([density 192 | transmittance 192 |
 * phase 192], log-encoded as the reference does), dev_aux = n x 5 fp32
 * (g, gamma, srp.x, srp.y, srp.z), dev_out = n x 3 fp32. */
int mr_radiance_predict(const mr_network* net, int32_t precision, const float* dev_desc,
                        const float* dev_aux, int32_t n, float* dev_out, void* stream);

/* Descriptor gather (core/radiancePredict.cu:319-368) for n points:
 * dev_pos n x 3, dev_frame n x 12 (XMain, YMain, ZMain, LXMain), writes
 * dev_desc n x 576 and dev_aux n x 5 (g, gamma, srp) for the given alpha, g,
 * scatter_rate. Volume tables must be up to date. */
int mr_gather_descriptors(const mr_volume* v, const mr_network* net, const float* dev_pos,
                          const float* dev_frame, int32_t n, float alpha, float g,
                          mr_float3 scatter_rate, float* dev_desc, float* dev_aux, void* stream);

/* Seeded procedural cloud (benchmark / training input): Perlin fBm with
 * `octaves` octaves from `base_freq`, lacunarity and gain, normalised to
 * [0,1], thresholded at `threshold` and shaped by a radial falloff; res^3
 * fp32 into dev_out, index (x*res+y)*res+z. */
int mr_generate_cloud(int32_t res, uint32_t seed, int32_t octaves, float base_freq, float lacunarity,
                      float gain, float threshold, float* dev_out, void* stream);
/* The 256-entry noise permutation the cloud generator uses for `seed`. */
int mr_cloud_permutation(uint32_t seed, int32_t* host_out256);

/* Self-test of the tensor-core tile path (no reference counterpart): one
 * 128 x n x k BF16 product D = A * B^T through the same shared-memory and
 * instruction descriptors as the network kernel. host_a 128 x k and host_b
 * n x k are BF16 bit patterns, row-major; host_d receives 128 x n fp32.
 * Shapes (n, k): (16,16) (32,32) (16,32) (32,64) (64,128) (128,128). */
int mr_tc_selftest(int32_t n, int32_t k, const uint16_t* host_a, const uint16_t* host_b, float* host_d);
/* The same tile product with E4M3 operands (kind::f8f6f4, no reference
 * counterpart): host_a 128 x k and host_b n x k are E4M3 bytes, row-major.
 * Shapes (n, k): (16,32) (32,32) (64,128) (128,128). */
int mr_tc_selftest_fp8(int32_t n, int32_t k, const uint8_t* host_a, const uint8_t* host_b, float* host_d);
/* The same tile product with fp32 operands on the TF32 path (kind::tf32, no
 * reference counterpart): host_a 128 x k and host_b n x k fp32, row-major.
 * split != 0: each operand is split into a TF32 part and an fp32 remainder
 * and D sums three TF32 products (A_hi B_hi + A_hi B_lo + A_lo B_hi), which
 * carries about 22 bits of the product; split == 0: one TF32 product.
 * Shapes (n, k): (16,16) (32,32) (32,64) (64,128). */
int mr_tc_selftest_tf32(int32_t n, int32_t k, const float* host_a, const float* host_b, float* host_d,
                        int32_t split);
/* Self-test of the exact sampler's two forms (no reference counterpart): for
 * n points uv (host_uv, n x 3, texture space) over one
 * MR_SAMPLER_SELFTEST_RES^3 fp32 table (host_table, index (x*R+y)*R+z),
 * host_out (n x 6) receives the trilinear border-0 filter from texel loads and
 * from texture gathers, the trilinear clamp filter from loads and gathers, and
 * the bilinear clamp filter of the table's first R x R values at (uv.x, uv.y)
 * from loads and gathers. The two forms agree bit for bit except where a
 * texel is subnormal (the texture unit reads those as 0). */
#define MR_SAMPLER_SELFTEST_RES 32
int mr_sampler_selftest(int32_t n, const float* host_table, const float* host_uv, float* host_out);
/* Failure path of the kernels' bounded waits (no reference counterpart): one
 * CTA allocates tensor memory, waits with a limit of limit_us (1 .. 10^6) on an
 * mbarrier that nothing arrives on, records the timeout and frees the tensor
 * memory. Returns MR_ERR_TIMEOUT (the expected outcome) with the time the wait
 * took in *host_waited_ns (may be NULL); the device stays usable. */
int mr_tc_wait_selftest(int32_t limit_us, int64_t* host_waited_ns);
/* BF16 tile product D[128 x n] = A[128 x k] B[n x k]^T (row-major inputs)
 * with A (a_mn = 1) and / or B (b_mn = 1) read MN-major: stored in the
 * canonical K-major layout of the transpose, as the BF16 training reads its
 * forward tiles and weights in the backward products. Shapes (n, k):
 * (64, 32), (128, 64), (128, 128), (64, 128). */
int mr_tc_selftest_mn(int32_t n, int32_t k, int32_t a_mn, int32_t b_mn, const uint16_t* host_a,
                      const uint16_t* host_b, float* host_d);
/* Memory-path probe (no reference counterpart): reads dev_buf (`bytes`, a
 * multiple of 16, 16-byte aligned) `passes` times with 16-byte loads that
 * bypass L1, from a resident grid; dev_sink is one device word. Time it with
 * events on `stream`: a buffer that fits in L2 gives the L2 read bandwidth, a
 * buffer far larger than L2 the HBM read bandwidth. */
int mr_stream_read_probe(const void* dev_buf, size_t bytes, int32_t passes, uint32_t* dev_sink, void* stream);
/* Error word of the tensor-core network kernel of `net` (an mbarrier wait
 * that timed out): MR_ERR_TIMEOUT if set; `reset` clears it. */
int mr_network_check(const mr_network* net, int32_t reset);

/* Neural render into a fixed scratch (no reference counterpart): the same
 * trace / gather / network passes as mr_render with MR_RT_MRPNN, but the
 * per-pixel records and descriptor columns live in a module-resident device
 * array of MR_NOALLOC_SCRATCH_MIB MiB instead of the volume's growable
 * scratch, so the call allocates no device or host memory.
 *  - width*height must be <= MR_NOALLOC_MAX_PIXELS (else MR_ERR_ARG);
 *  - sampler must be MR_SAMPLER_EXACT (texture tables are allocated on first
 *    use), precision FP32 or BF16;
 *  - the HG table and transmittance pyramid must already be built for p's g,
 *    seed, light and alpha (mr_volume_update_hglut / _update_tr, or an
 *    earlier mr_render): MR_ERR_STATE otherwise;
 *  - the scratch is one per device and process: overlapping calls (several
 *    streams or threads on one device) race on it and must be serialised by
 *    the caller;
 *  - the first call on a device looks the scratch address up (and may load
 *    the module there), so make it before any stream capture;
 *  - the array belongs to the module of every neural-render kernel: loading
 *    that module on a device (any neural render there) holds its
 *    MR_NOALLOC_SCRATCH_MIB MiB of device memory for the life of the process,
 *    whether or not this entry point is ever called.
 * Stage timing (mr_volume_set_timing) does not cover this call. */
#define MR_NOALLOC_MAX_PIXELS 16384
#define MR_NOALLOC_SCRATCH_MIB 45
int mr_render_neural_noalloc(mr_volume* v, const mr_network* net, const mr_render_params* p, float* dev_rgb,
                             void* stream);

/* ---- interactive rendering (VolumeRender::Render(float3*, Histogram*, unsigned*, ...),
 *      core/volume.cu:469-547, with RenderCamera / Denoise / ReprojectionDenoise
 *      core/volume.cu:57-145,181-295) ------------------------------------------- */

/* Histogram (core/volume.hpp:12-19): 10 bins per channel of x / (1 + x), the
 * sample count, and running means of l^2 and l, l = sum over channels of
 * x / (1 + x). In the neural mode the three scalars hold the previous
 * frame's colour (the reference's reprojection history). */
typedef struct {
  float bin[30];
  float total_samples;
  float x2;
  float x;
} mr_histogram;

/* Per-frame settings of the interactive path. */
typedef struct {
  mr_float3 prev_ori, prev_up, prev_right; /* camera of the previous frame (neural reprojection) */
  int32_t frame_index;  /* randseed / frameNum: 0 restarts the accumulation; also the sample index */
  int32_t checkerboard; /* SetCheckboard: delta tracking renders half the pixels per frame,
                           alternating with frame_index parity */
  int32_t tone;         /* 0 none, 1 gamma 2.2, 2 ACES */
  int32_t denoise;      /* histogram-weighted 11 x 11 filter (delta tracking) */
  float exposure;       /* SetExposure */
} mr_interactive;

/* One interactive frame. PT: one delta-tracking sample per (rendered) pixel
 * blended into dev_accum (W*H*3 running mean) and the histograms (W*H), then
 * Denoise into dev_bgra (W*H, 0xAARRGGBB). MRPNN: the neural render of this
 * frame blended with the previous frame's colour at the reprojected pixel
 * (dev_hist holds the history), then tone mapped and packed. Buffers are the
 * caller's device memory; rows are top-first like mr_render. */
int mr_render_interactive(mr_volume* v, const mr_network* net, const mr_render_params* p, const mr_interactive* it,
                          float* dev_accum, mr_histogram* dev_hist, uint32_t* dev_bgra, void* stream);
/* Denoise<denoise> (core/volume.cu:210-264) alone: filter, exposure, tone map
 * and pack of an accumulated image and its histograms. */
int mr_denoise(const float* dev_accum, const mr_histogram* dev_hist, uint32_t* dev_bgra, int32_t width,
               int32_t height, const mr_interactive* it, void* stream);

/* ---- batched neural rendering (no reference counterpart: the reference renders
 *      one volume and one view per call, core/volume.cu:410-467) ---------------- */

typedef struct mr_batch mr_batch;

/* A batch of (volume, view) jobs rendered together: the jobs' pixels are one
 * flattened space processed in waves (one batched trace, gather and network
 * launch per wave over all jobs' records). Every job is MR_RT_MRPNN; all
 * share one precision and sampler; jobs on one volume must share its light,
 * alpha, g and seed (each volume holds one set of tables). */
int mr_batch_create(mr_batch** out);
int mr_batch_destroy(mr_batch* b);
/* Adds a job: p as for mr_render; dev_rgb = width*height*3 floats. Its
 * sample index starts at p->sample_offset and advances by one per frame. */
int mr_batch_add(mr_batch* b, mr_volume* v, const mr_render_params* p, float* dev_rgb);
/* Builds the jobs' tables, uploads the job table and allocates the wave
 * scratch (wave_pixels 0 = min(total, 4 Mi)). Must follow the last add. */
int mr_batch_prepare(mr_batch* b, const mr_network* net, int64_t wave_pixels, void* stream);
/* Times full frames over wave sizes 1/2/4 Mi pixels, then the trace and
 * gather block sizes 64/128/256, keeps the fastest and reports them. The
 * timed frames advance the jobs' sample indices. */
int mr_batch_autotune(mr_batch* b, const mr_network* net, int64_t* host_wave, int32_t* host_trace_block,
                      int32_t* host_gather_block, void* stream);
/* Renders one frame of every job (stream-ordered launches). */
int mr_batch_render(mr_batch* b, const mr_network* net, void* stream);
/* Captures one frame of the batch into a CUDA graph on `stream` (not the
 * legacy default stream); renders one eager frame first. */
int mr_batch_capture(mr_batch* b, const mr_network* net, void* stream);
/* Replays the captured graph: one more frame of every job. */
int mr_batch_launch(mr_batch* b, void* stream);
/* Per-frame completion times (no reference counterpart). With timing on,
 * every batch frame (eager or a replay captured after this call) records the
 * device timer before its first launch and after each wave; the jobs' pixels are
 * laid out in the order they were added, so a job's frame is complete when
 * the wave holding its last pixel is. Call after mr_batch_prepare / _autotune
 * and before mr_batch_capture (it drops a captured graph). */
int mr_batch_set_timing(mr_batch* b, int32_t enable);
/* Milliseconds from the start of the last batch frame to the completion of
 * each job's frame (n = number of jobs, in add order), from the device's
 * global timer (about 1 us resolution); waits for the device. */
int mr_batch_frame_times(mr_batch* b, float* host_ms, int32_t n);
/* Counters of the frames since mr_batch_prepare's last reset: [0] density
 * fetches, [2] loop-cap hits, [3] active pixels (of the last frame). */
int mr_batch_counters(const mr_batch* b, uint64_t* host_out4);

/* ---- training (replaces dataGen.cu and the offline training of NNWeight.cuh) --- */

typedef struct mr_trainer mr_trainer;

/* MeanFreePathSample / GetDesiredCountSample (dataGen.cu:148-216): n_rays rays
 * from the sphere of radius 0.5 towards the volume, up to four Woodcock
 * vertices each (extinction scale alpha, HG g), jittered by up to 1/128 and
 * paired with the primary or current ray direction as the reference does.
 * Writes up to `cap` points (dev_pos, dev_dir: cap x 3) and their number. */
int mr_train_points(mr_volume* v, float alpha, float g, uint32_t seed, int32_t n_rays, int32_t cap, float* dev_pos,
                    float* dev_dir, int32_t* host_count, void* stream);
/* GetSamples (core/volume.cu:550-626, core/render.cuh:276-315): training
 * labels, the multiple-scattering radiance at each point along its view
 * direction for light L (unit intensity), albedo and g, over `spp` paths of at
 * most max_bounces vertices. Adds the FP64 radiance sums to dev_sum (n
 * doubles, caller-zeroed); label = sum / spp. */
int mr_train_labels(mr_volume* v, const float* dev_pos, const float* dev_dir, int32_t n, mr_float3 light_dir,
                    float alpha, float g, float albedo, int32_t max_bounces, int32_t spp, uint32_t seed,
                    double* dev_sum, void* stream);
/* The random view / light frames NNPredict draws (core/render.cuh:355-369) for
 * n view directions: dev_frame n x 12 (X, Y, Z, LX) for mr_gather_descriptors. */
int mr_train_frames(const float* dev_dir, int32_t n, mr_float3 light_dir, uint32_t seed, float* dev_frame,
                    void* stream);
/* A trainer holds fp32 master weights (blob layout), Adam moments and a
 * gradient buffer. The loss of a row is (X - log(1 + label / srp.x))^2, X the
 * head output of the first albedo channel (the network predicts
 * max(exp(X) - 1, 0) * srp); the step loss is its mean over the n rows.
 * dev_desc n x 576 and dev_aux n x 5 as mr_gather_descriptors writes them. */
int mr_trainer_create(const float* host_weights, size_t count, mr_trainer** out);
int mr_trainer_destroy(mr_trainer* t);
/* Gradient of the mean loss (MR_WEIGHT_TOTAL floats) without updating. */
int mr_trainer_gradient(mr_trainer* t, const float* dev_desc, const float* dev_aux, const float* dev_label,
                        int32_t n, float* host_grad, float* host_loss, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected) at rate lr;
 * host_loss (optional) receives the batch loss before the update. */
int mr_trainer_step(mr_trainer* t, const float* dev_desc, const float* dev_aux, const float* dev_label, int32_t n,
                    float lr, float* host_loss, void* stream);
int mr_trainer_weights(const mr_trainer* t, float* host_out, size_t count);
/* Arithmetic of the training step: MR_PREC_FP32 (default; every layer on the
 * CUDA cores, one row per thread) or MR_PREC_BF16: the head's LC0 / LC1 / LC2
 * forward, input-gradient and weight-gradient products as tcgen05 MMAs with
 * BF16 operands and FP32 accumulation, the rest in FP32; Adam keeps the FP32
 * master weights either way. */
int mr_trainer_set_precision(mr_trainer* t, int32_t precision);

/* Wait for `stream` with a watchdog: MR_ERR_TIMEOUT after timeout_ms. */
int mr_sync(void* stream, int32_t timeout_ms);

/* Per-stage CUDA-event timing of this volume's kernels (off by default).
 * Stages: 0 delta tracking, 1 neural trace, 2 neural descriptor gather,
 * 3 TR build, 4 HG table build, 5 pyramid build, 6 neural network (MLP),
 * 7 the fp32 network's main-trunk kernel alone (part of stage 6).
 * mr_volume_stage_times waits
 * for the device, returns the summed milliseconds and launch counts of the
 * first n stages since the last query, and resets them. */
int mr_volume_set_timing(mr_volume* v, int32_t enable);
int mr_volume_stage_times(mr_volume* v, double* host_ms, int32_t* host_launches, int32_t n);

/* Counters of the last render on this volume: [0] density fetches, [1] paths,
 * [2] loop-cap hits, [3] active neural pixels. */
int mr_volume_counters(const mr_volume* v, uint64_t* host_out4);

#ifdef __cplusplus
}
#endif

#endif /* MRPNN_B200_H */
