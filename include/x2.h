/*
 * x2 — C ABI of the B200 path-sample engine (libx2.so).
 *
 * The reference has no C ABI for this path: it sits behind two C++ interfaces, the per-sample
 * `integrate<Backend>(const mixed::Config&, U32 pixel, U32 index, Backend&, Radiance&)`
 * (xpu2/interactive/async_integrator.h:3047) and the per-lane `GpuLane`
 * (xpu2/interactive/async_gpu.h:82, begin/launch/poll/downloadFilm/sums/counts at :1372-1707).
 * Every entry point below names the reference interface it replaces.
 *
 * Conventions: plain C, status codes are int (X2_OK = 0). Handles are owned by the library; the caller
 * owns every array it passes. No callbacks. One context is used from one host thread. Calls are
 * asynchronous on the context's CUDA stream except where a comment says they wait; waits are bounded.
 */
#ifndef X2_H
#define X2_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference reports failures as cpu::need -> std::runtime_error on the host and as
 * SampleStatus::Error / DeviceState::errors on the device (async_gpu_abi.h:45); here they are codes. */
enum {
    X2_OK = 0,
    X2_EINVAL = 1,    /* a bad argument: null pointer, size out of range, config the engine does not admit */
    X2_ECUDA = 2,     /* a CUDA runtime error (x2_last_error has the text) */
    X2_ENOMEM = 3,    /* a device or host allocation failed */
    X2_ETIMEOUT = 4,  /* a bounded wait gave up */
    X2_EAUDIT = 5,    /* the per-pixel sample-count audit failed (async_render.h:1036-1039) */
    X2_ENODEV = 6,    /* no CUDA device */
    X2_EDEVICE = 7    /* the device reported errors (sample errors, a traversal stack overflow) */
};

/* Per-sample outcome, SampleStatus in async_integrator.h:35 (same values). */
enum { X2_DONE = 0, X2_MISS = 1, X2_ERROR = 2, X2_SKIP = 3, X2_DEFER = 4 };

/* sample::Identity (sample_stream.h:42): 32-bit pixel, 64-bit sample index, stream (frame seed) and branch. */
typedef struct x2_identity {
    uint32_t pixel;
    uint32_t pad;
    uint64_t index, stream, branch;
} x2_identity;

/* The unit of work, async::Chunk (async_integrator.h:3057-3063): one 8x8 tile and a sample range. 16 bytes. */
typedef struct x2_chunk {
    uint32_t tile, first, count, cell;
} x2_chunk;

/* Pixel filters, surface::Filter (surface_core.h:24). */
enum { X2_FILTER_BOX = 0 };

/* Materials admitted: the UsdPreviewSurface subset (shade_material.h:338-383) with useSpecularWorkflow = 1.
 * LAMBERT: diffuseColor = diffuse, specularColor black -> one Lambert lobe (shade_builder.h:689-697).
 * GGX: the Schlick specular path (MatModoUsdSpecular; shade_builder.h:541-556): one GGX lobe whose Fresnel is
 * Schlick with F0 = specular, plus a Lambert lobe under it only when diffuse is not black (not admitted: keep it
 * black). emission is emissiveColor (addEmission).
 * diffuse_texture: 0 none; k + 1 binds the scene's texture k to diffuseColor as a UsdUVTexture read at the mesh's
 * st primvar (a UsdPrimvarReader of the vertices' uvs; shade_mapnodes.h:972-997, :1012-1030): the texel multiplies a
 * non-black diffuse (MapBinding BindColor, shade_maps.h). */
enum { X2_MAT_LAMBERT = 0, X2_MAT_GGX = 1 };
typedef struct x2_material {
    uint32_t kind;
    float diffuse[3];
    float specular[3];
    float emission[3];
    float roughness;
    uint32_t diffuse_texture;
} x2_material;

/* A texture: one level of fp32 RGB texels, row-major, row 0 the image's top (a lookup at st reads row (1 - t) x
 * height, texture_core.h lookup), wrap 1 periodic, 0 clamped. UsdUVTexture reads it with no filter footprint
 * (MoonRay sets the derivatives to zero): level 0 only, bilinear on primary paths and the closest texel on indirect
 * ones (texture_core.h bilinear, closest; shade_mapnodes.h textureMode). */
typedef struct x2_texture {
    uint32_t width, height, wrap, pad;
    const float* rgb;
} x2_texture;

/* Lights admitted: lights::Light (light_core.h:59-117) of type Env (constant, whole sphere or hemisphere, no
 * image), Rect (no image, no spread, no clear radius) and Distant (no image: a cone of half-angle acos(cos_theta_max)
 * about -direction, sampled uniformly; inv_area = 1 / (2 pi versine_theta_max)). Linear parts are rows, as the
 * reference stores them. */
enum { X2_LIGHT_ENV = 0, X2_LIGHT_RECT = 1, X2_LIGHT_DISTANT = 4 };
enum { X2_SIDE_REGULAR = 0, X2_SIDE_REVERSE = 1, X2_SIDE_TWO = 2 };
typedef struct x2_light {
    uint32_t type, sidedness, visible_in_camera, hemispherical;
    float radiance[3];
    float position[3], direction[3];  /* local origin; local +Z (the lit side of a one-sided rect), unit */
    float local2render[3][3];         /* rows, with scale */
    float render2local[3][3];         /* its inverse (rows) */
    float render2local_rot[3][3];     /* rotation only (rows) */
    float scale, inv_area, plane_offset, half_width, half_height;
    uint32_t visibility_mask;         /* rdl2 VisibilityType bits of the lobes that see it (0xfc: all) */
    float cos_theta_max, versine_theta_max;  /* Distant: the cone's half-angle cosine, 1 - that */
} x2_light;

/* Participating media: volume::Shader (volume_core.h:64-111) of kind VDB (a VdbVolume) whose density (and, when it
 * glows, emission) are dense grids, bound to an axis-aligned box (its closed mesh: two triangles a face, outward
 * normals; rays cross it at entry and exit as the reference's volume crossings do, async_cpu.h:1089-1149).
 * Extinction = gain x density (interpolation: 0 point, 1 box/trilinear, 2 quadratic; shadows read the nearest voxel),
 * albedo = color_mult, emission = incandescence x the emission grid's nearest voxel, Henyey-Greenstein g. */
typedef struct x2_volume {
    float bound_lo[3], bound_hi[3];
    uint32_t density_grid, emission_grid;  /* grid indices (emission: ~0u none) */
    uint32_t interpolation;
    float feature_size;                    /* the march's step unit: the cube root of a voxel's volume */
    float world_to_grid[12];               /* rows of an affine map (x, y, z, translation), render -> grid space */
    float gain[3], color_mult[3], incandescence[3];
    float g;
    uint32_t light_set;                    /* lights that light it: bit i light i (~0u all) */
    float surface_opacity_threshold;
} x2_volume;

/* A dense grid of float (channels 1) or float3 (channels 3) voxels: dims from index lo, x fastest; zero outside.
 * world_to_index: OpenVDB's linear world-to-index map, a row-vector 4x4 in doubles (volume_grid.h:33-47). */
typedef struct x2_grid {
    uint32_t channels;
    int32_t lo[3], dims[3];
    double world_to_index[16];
    const float* values;
} x2_grid;

/* surface::Camera's perspective subset (surface_core.h:93-115): row-vector matrices, clip planes. */
typedef struct x2_camera {
    float raster_to_camera[4][4];
    float camera_to_render[4][4];
    float near_clip, far_clip;
} x2_camera;

/* A scene: triangles grouped by mesh (geom), meshes contiguous in triangle order; each mesh one material.
 * Vertices are fp32 (3 a vertex), triangles 3 vertex indices each. mesh_first has mesh_count + 1 entries. */
typedef struct x2_scene_desc {
    uint32_t vertex_count, triangle_count, mesh_count, material_count, light_count, pad;
    const float* vertices;
    const uint32_t* triangles;
    const uint32_t* mesh_first;
    const uint32_t* mesh_material;
    const x2_material* materials;
    const x2_light* lights;
    x2_camera camera;
    uint32_t volume_count, grid_count;  /* volume_count <= 32 */
    const x2_volume* volumes;
    const x2_grid* grids;
    /* Textures and texture coordinates: uvs null (no mesh has st) or 2 floats a vertex (MeshAttributes uvs at
     * RateVertex, shade_material.h:143-153). */
    uint32_t texture_count, pad2;
    const x2_texture* textures;
    const float* uvs;
} x2_scene_desc;

/* mixed::Config (gpu_jobs.h:10-44), the fields this engine reads, field for field with the same defaults
 * (x2_config_defaults). Policy 15 and the shadow-reuse mask are what mixed::config (cpu_jobs.h:8-27) sets for
 * the path tracer. */
typedef struct x2_config {
    uint32_t width, height, seed, spp, sampling;
    uint32_t filter;
    float filter_width;
    uint32_t light_count, bsdf_samples, light_samples, max_depth, max_diffuse_depth, clamp_depth;
    float rr_threshold, clamp_value;
    uint32_t max_glossy_depth, max_mirror_depth, max_hair_depth, max_presence_depth, shadow_terminator_fix;
    float roughness_clamping, transparency_threshold;
    uint32_t visible_lights;
    float presence_threshold, presence_quality;
    uint32_t shadow_reuse;
    /* Volumes (gpu_jobs.h:18-28): how many (the scene's), MoonRay's volume scene variables. */
    uint32_t volume_count, max_volume_depth, volume_illumination_samples, volume_overlap_mode;
    float volume_transmittance_threshold, volume_attenuation_factor, volume_contribution_factor, volume_phase_attenuation_factor;
    float inv_volume_quality, inv_volume_shadow_quality;
    /* The volume integrals' estimator: 0 the reference's decoupled ray marching (per-sample parity with the
     * reference); 1 delta and ratio tracking over 32^3 majorant grids (no reference counterpart: the same integrals
     * sampled otherwise; grey extinction, max_volume_depth 1, overlap modes sum or max). */
    uint32_t volume_estimator;
    uint32_t reserved[7];
} x2_config;

/* Ray counters, the reference's XPU2_PROFILE ray counts (async_gpu_abi.h:16-20): hit rays (trace), shadow rays
 * of light samples (NEE) and of BSDF samples, and the bounces that stood for a shadow ray (held). */
typedef struct x2_counters {
    uint64_t trace, shadow_nee, shadow_bsdf, held, samples, errors, stack_overflows, pad;
} x2_counters;

/* A finished launch, GpuLane's Completion (async_gpu.h:65-71). */
typedef struct x2_completion {
    uint64_t launch;      /* its sequence number */
    uint64_t samples;     /* samples finished (Done or Skip) */
    uint64_t errors;      /* samples that ended in Error */
    float milliseconds;   /* device time of the launch (CUDA events on the context's stream) */
    uint32_t pad;
} x2_completion;

typedef struct x2_ctx x2_ctx;
typedef struct x2_scene x2_scene;

/* ---- library ---- */
const char* x2_version(void);
const char* x2_last_error(void);        /* text of the last failure on this thread */
void x2_config_defaults(x2_config* c);  /* mixed::Config's defaults (gpu_jobs.h:11-44) plus the path tracer's */

/* ---- context: replaces GpuLane's construction (async_gpu.h:82) ---- */
int x2_open(int device, x2_ctx** out);
int x2_close(x2_ctx* ctx);
int x2_synchronize(x2_ctx* ctx, int timeout_ms);  /* waits (bounded) for the context's stream */

/* ---- sampler test API: sample::samplingWord (sample_stream.h:127-144) for n identities/dimensions ---- */
int x2_sample_words(x2_ctx* ctx, const x2_identity* ids, const uint32_t* dims, uint64_t n, uint32_t policy,
                    uint32_t* out);                      /* host arrays; waits */
int x2_sample_words_device(x2_ctx* ctx, const x2_identity* d_ids, const uint32_t* d_dims, uint64_t n,
                           uint32_t policy, uint32_t* d_out);  /* device arrays; asynchronous */

/* ---- scene: replaces the plan upload of GpuLane (cpu::Plan -> device records) ---- */
int x2_scene_load(x2_ctx* ctx, const x2_scene_desc* desc, x2_scene** out);  /* builds the BVH on the device */
int x2_scene_free(x2_scene* scene);
int x2_config_set(x2_scene* scene, const x2_config* config);  /* mixed::config(plan) */
int x2_scene_info(x2_scene* scene, uint64_t* bvh_nodes, uint64_t* bvh_bytes, uint64_t* triangle_bytes,
                  float* build_ms);

/* ---- per-sample API: integrate() (async_integrator.h:3047) for n (pixel, index) pairs ----
 * pairs: 2n uint32 (pixel, index); rgba: 4n doubles (Radiance rgb + alpha); status: n SampleStatus. */
int x2_integrate(x2_scene* scene, const uint32_t* pairs, uint64_t n, double* rgba, uint32_t* status); /* waits */
int x2_integrate_device(x2_scene* scene, const uint32_t* d_pairs, uint64_t n, double* d_rgba, uint32_t* d_status);

/* ---- traversal API: Backend::trace / Backend::visible (async_cpu.h:669-720, :944-967; async_gpu_device.h:298-355,
 * 521-533) for n rays, 8 floats each (origin xyz, direction xyz, near, far): the closest hit's scene triangle
 * (~0u: none) and t, and whether anything occludes [near, far]. ---- */
int x2_trace_rays(x2_scene* scene, const float* rays, uint64_t n, uint32_t* tri, float* t, uint32_t* occluded); /* waits */
int x2_trace_rays_device(x2_scene* scene, const float* d_rays, uint64_t n, uint32_t* d_tri, float* d_t, uint32_t* d_occluded);

/* ---- lane API: GpuLane::begin/launch/poll/downloadFilm/sums/counts (async_gpu.h:1372-1707) ---- */
int x2_frame_begin(x2_scene* scene, uint32_t samples_per_chunk);          /* begin(): clears the film */
int x2_launch(x2_scene* scene, const x2_chunk* chunks, uint32_t count);   /* launch(): host chunks */
int x2_poll(x2_scene* scene, x2_completion* out);  /* poll(): 1 and *out when a launch finished, 0 if none */
int x2_wait(x2_scene* scene, int timeout_ms, x2_completion* out);  /* waits for every launch in flight */
int x2_render_frame(x2_scene* scene, uint32_t first, uint32_t count);  /* every tile, samples [first, first+count) */
/* The wavefront form of a launch (no counterpart in the reference, whose wavefront was ruled out,
 * xi/INDEXER.md:161-181): the same samples as x2_launch, by compacted extend / shade / shadow kernels with path
 * regeneration; the same film. The launch is one CUDA graph whose iterations run in a conditional while node until no
 * path is left (at most a bound from the items, paths and depth; a launch past it completes with X2_EDEVICE at
 * x2_poll / x2_wait), so it returns without waiting, as x2_launch does. One BSDF sample a lobe (bsdf_samples = 1).
 * Paths in flight: x2_wavefront_reserve (default 2^23, halved while the path state a scene needs would pass 12 GB). x2_items_download reads the last wavefront launch's per-item radiance and
 * status (item = chunk * 64 * samples_per_chunk + position * samples_per_chunk + sample). */
int x2_wavefront_reserve(x2_scene* scene, uint32_t paths);
int x2_launch_wavefront(x2_scene* scene, const x2_chunk* chunks, uint32_t count);
int x2_render_frame_wavefront(x2_scene* scene, uint32_t first, uint32_t count);
int x2_items_download(x2_scene* scene, float* rgba, uint8_t* status, uint64_t n);  /* waits */
int x2_wavefront_info(x2_scene* scene, uint32_t* paths, uint32_t* records, uint32_t* iterations);
/* Per-kernel timing of wavefront launches (a diagnostic: no graph, a host sync an iteration). on: 1 on, 0 off, -1
 * unchanged; ms (5 floats, or null): the last timed launch's logic, extend, shade, shadow and film-reduce times. */
int x2_wavefront_timing(x2_scene* scene, int on, float* ms);
/* Wavefront launch shape (no reference counterpart; the autotuner's knobs). The results do not depend on it. */
typedef struct x2_wavefront_shape {
    uint32_t paths;          /* path slots in flight (0: 2^23, fewer when the launch has fewer items) */
    uint32_t refill;         /* 1..32 idle lanes that make a traversal warp fetch the next rays of its queue */
    uint32_t blocks_per_sm;  /* traversal and shade grids: blocks a SM, 1..32 */
    uint32_t trace_blocks;   /* traversal kernels' occupancy variant: blocks a SM their registers allow (0, 9, 10;
                                0: the compiler's choice) */
    uint32_t shade_blocks;   /* shade kernel's occupancy variant (0, 3, 4; with shade_split the lobe kernels at 4, or 5
                                when this is 5) */
    uint32_t tri_limit;      /* triangle tests a lane makes a traversal step, the rest on the next steps (1..32) */
    uint32_t batch_window;   /* x2_render_batch: work items a window (0: 2^27; at least one chunk a window) */
    uint32_t lobe_queues;    /* 1: shade takes the extended paths from per-lobe queues (GGX, Lambert, then none or
                                missed), sorted after extend, so a warp runs one lobe's code (surface scenes; volume
                                scenes are shaded in the extend queue's order either way); 0: in the extend queue's order */
    uint32_t shadow_order;   /* 1: the shadow queue by record (record k of every path together, mostly one light's rays
                                to neighbouring origins); 0: by path (each path's records together) */
    uint32_t extend_bins;    /* 1: the extend queue binned by the rays' direction octant (a warp's rays share their
                                children's near-to-far order); 0: in path-slot order */
    uint32_t short_stack;    /* 1: the traversal stacks' first 8 entries in shared memory; 0: all in local memory */
    uint32_t shade_split;    /* 1: shade as one kernel a per-lobe queue (GGX, Lambert, the rest; with lobe_queues 1, surface
                                scenes), each holding one lobe's code; 0: one shade kernel */
    uint32_t light_split;    /* 1, 2 (with shade_split): the GGX and Lambert vertices' light samples in kernels of their
                                own, after shade, from the vertex's stored inputs, at 6 (1) or 8 (2) blocks a SM; 0: inside
                                shade */
    uint32_t tri_overlap;    /* 1: a lane holding a leaf's triangles tests one a step and goes on visiting nodes meanwhile
                                (takes effect with short_stack 1 and trace_blocks below 9); 0: it visits no node until the
                                leaf is done */
} x2_wavefront_shape;
void x2_wavefront_shape_defaults(x2_wavefront_shape* shape);
int x2_wavefront_tune(x2_scene* scene, const x2_wavefront_shape* shape);
/* The autotuner: times wavefront launches of `tiles` evenly spaced tiles (0: all) at `spp` samples, one knob at a time
 * (paths, refill, tri_limit, shade_blocks, trace_blocks, blocks_per_sm, lobe_queues, shadow_order, extend_bins,
 * short_stack, shade_split, light_split; best of two launches a candidate), sets the
 * fastest shape and returns it (best, best_ms may be null). Renders into the scene's film, which it leaves reset (as
 * x2_frame_begin(scene, spp)). Waits. */
int x2_wavefront_autotune(x2_scene* scene, uint32_t tiles, uint32_t spp, x2_wavefront_shape* best, float* best_ms);
/* Batched renders (no reference counterpart; the reference renders one plan a lane): a request is one scene's frame,
 * samples [first, first + count) of every pixel, at the scene's own config (resolution, depth, lights, frame seed). */
typedef struct x2_request {
    x2_scene* scene;
    uint32_t first, count;  /* count 1..2^21 */
} x2_request;
/* Renders n requests (1..256; distinct scenes of ctx, each configured with bsdf_samples = 1) in one wavefront
 * launch: path slots shared by all requests and regenerated across them, each path in its own scene; the first
 * request's scene holds the path state and its launch shape (x2_wavefront_tune) applies. Each scene's film is reset
 * first (as x2_frame_begin(scene, count)) and then holds exactly the film x2_launch_wavefront gives for all its
 * tiles; x2_film_download / x2_audit read it. Waits. out (or null): samples and errors of the whole batch, its device
 * milliseconds; the ray counters go to the first scene's x2_counters. */
int x2_render_batch(x2_ctx* ctx, const x2_request* requests, uint32_t n, x2_completion* out);
/* ---- adaptive sampling (async_render.h's adaptive frame; async_adaptive.h, async_adaptive.cu) ----
 * A frame whose film also keeps the odd-index sums (GpuLane::begin's adaptive frame, async_gpu.h:1372): as
 * x2_frame_begin. */
int x2_frame_begin_adaptive(x2_scene* scene, uint32_t samples_per_chunk);
/* One step of the reference's GPU pass chain (async_adaptive.cu chainErrors, chainTrees, chainMasks) on the current
 * adaptive film: each pixel's error (pixelError, async_integrator.h:3109), the overlapping regions' trees
 * (async_adaptive.h Tree, Regions; target error `target`), and each 8x8 tile's mask of the pixels the next pass of
 * `size` samples takes (uniform: every pixel in the image, no trees); each active pixel's first sample index and
 * planned count move on. errors (a float a pixel), masks (a uint64 a tile, bit y * 8 + x) and stop (1: every region
 * converged, the chain stops) are host arrays, each may be null. Waits. */
int x2_adaptive_step(x2_scene* scene, float target, uint32_t uniform, uint32_t size, float* errors, uint64_t* masks, uint32_t* stop);
typedef struct x2_adaptive_result {
    uint32_t passes, converged;  /* passes rendered; 1 when every region converged before the schedule ran out */
    uint64_t samples;            /* samples rendered */
    float milliseconds;          /* host time of the whole frame */
    uint32_t pad;
} x2_adaptive_result;
/* An adaptive frame (the reference's adaptive frame with its GPU chain, async_render.h / async_gpu.h:1929-2090):
 * MoonRay's pass schedule for max_samples (one sample, then 4, 6, 8, ... more), passes starting below min_samples
 * uniform, then after each pass the chain's errors, trees and masks; each pass renders its active tiles' masked pixels
 * in the wavefront form, each pixel from its own next sample index. Ends when every region has converged (target
 * error), a pass has no active pixel, or the schedule runs out. The whole frame is queued on the device at once (one
 * graph: the chain, the active tiles' compaction and each pass's launch), so no pass waits on the host. The film (sums,
 * odd sums, counts) is then read as after any launch; x2_adaptive_planned gives each pixel's planned count (for
 * x2_audit). Waits. */
int x2_render_adaptive(x2_scene* scene, uint32_t min_samples, uint32_t max_samples, float target, x2_adaptive_result* result);
/* The same frame with cellular generations in place of MoonRay's trees (the reference's preview default,
 * adaptive::Cellular, async_adaptive.h:147-232): before each adaptive pass the image's 8x8 tiles are a generation of
 * cells, a tile living by its error over the target and its live neighbours; a live tile samples all its pixels. Ends
 * when a generation has no live tile or the schedule runs out. Waits. */
int x2_render_adaptive_cellular(x2_scene* scene, uint32_t min_samples, uint32_t max_samples, float target, x2_adaptive_result* result);
/* A frame by sampling generations under a budget of samples (cpu::Plan sampleBudget with budgetBySamples): the
 * cellular generations, each with the target the samples still to spend would bring every tile to (no lower than
 * floor; 0: none), made on the host between passes as the reference makes them (async_render.h:1318-1410); a pass
 * whose live tiles want more than is left takes those furthest above the target first. Ends once the budget is spent,
 * a generation has no live tile or the schedule runs out. Waits. */
int x2_render_adaptive_budget(x2_scene* scene, uint32_t min_samples, uint32_t max_samples, float floor, uint64_t budget,
                              x2_adaptive_result* result);
int x2_adaptive_planned(x2_scene* scene, uint32_t* planned);

/* ---- the work grid: replaces Grid (async_grid.h:96-430) as the GPU lane uses it (GridOptions::mode 1, every cell
 * the GPU's), and the GPU feeder's claims (async_render.h:600-605, 780-797) ----
 * The image in square cells, each handing out its chunks (x2_chunk.cell: the chunk's cell) through one cursor, so any
 * number of claimants take each chunk exactly once. A uniform frame's chunks: its sample ranges (progressive: 1, 1, 2,
 * then samples_per_chunk samples; else samples_per_chunk each) over every tile with pixels in the viewport, each
 * cell's ordered by range and then tile; a claim reaches no further than the frontier (the least range still
 * unclaimed among the cells with work left), an important cell one range further. The CPU lane's side of the
 * reference's grid (owners, rights of passage, rates, suitability, ownership across frames) has no counterpart: the
 * product has no CPU lane. Claims are thread-safe; appends have one writer. */
typedef struct x2_workgrid x2_workgrid;
typedef struct x2_workgrid_options {
    uint32_t cell_size;          /* pixels, a multiple of 8 (default 64) */
    uint32_t samples_per_chunk;  /* sample indices a chunk (default 4) */
    uint32_t progressive;        /* 1: the progressive order (default); 0: ranges of samples_per_chunk */
    uint32_t sample_first, sample_count; /* a share of the frame: its sample indices [first, first + count) (count 0: all) */
    uint32_t workers;            /* the broker's cellular workers, each a share of a launch (default 32) */
} x2_workgrid_options;
void x2_workgrid_options_defaults(x2_workgrid_options* options);
/* A grid for a width x height frame of spp samples. empty: no chunks made (cells filled by x2_workgrid_append).
 * viewport: min x, min y, max x, max y (half open; null: the image). */
int x2_workgrid_create(uint32_t width, uint32_t height, uint32_t spp, const x2_workgrid_options* options, uint32_t empty,
                       const int32_t* viewport, x2_workgrid** out);
void x2_workgrid_free(x2_workgrid* grid);
int x2_workgrid_info(const x2_workgrid* grid, uint32_t* width, uint32_t* height, uint32_t* spp, x2_workgrid_options* options);
uint32_t x2_workgrid_cells(const x2_workgrid* grid);
uint64_t x2_workgrid_total(const x2_workgrid* grid);  /* chunks published */
/* The frame's sample ranges: (first, count) pairs, up to capacity of them written; returns how many there are. */
uint32_t x2_workgrid_ranges(const x2_workgrid* grid, uint32_t* ranges, uint32_t capacity);
int x2_workgrid_cell(const x2_workgrid* grid, uint32_t cell, uint32_t* tiles, uint32_t* published, uint32_t* taken);
int x2_workgrid_append(x2_workgrid* grid, uint32_t cell, const x2_chunk* chunks, uint32_t n);
/* Up to n chunks of a cell, none past what the frontier allows; returns how many (0 once closed). */
uint32_t x2_workgrid_claim(x2_workgrid* grid, uint32_t cell, uint32_t n, x2_chunk* out);
uint32_t x2_workgrid_claimable(const x2_workgrid* grid, uint32_t cell);
uint32_t x2_workgrid_remaining(const x2_workgrid* grid, uint32_t cell);
uint32_t x2_workgrid_empty(const x2_workgrid* grid);
uint32_t x2_workgrid_frontier(const x2_workgrid* grid);
/* The cellular rules: the cell a worker in cell `current` (~0u: none) works next, ~0u when it may take nothing now
 * (Grid::choose); the starting cell of worker w of n (Grid::seed). */
uint32_t x2_workgrid_choose(const x2_workgrid* grid, uint32_t current, uint32_t salt);
uint32_t x2_workgrid_seed(const x2_workgrid* grid, uint32_t worker, uint32_t workers);
/* Important parts first: each cell's score (below zero: not known yet); cells above the mean are important. */
int x2_workgrid_set_scores(x2_workgrid* grid, const float* scores, uint32_t n);
void x2_workgrid_close(x2_workgrid* grid);  /* a drain: nothing is handed out any more */
/* Important parts first (async_render.h:1581-1611 cellScores, from the preview picture of async_cpu.h:1359-1379):
 * each cell's score from the scene's film so far, the mean over its sampled pixels of their tones' differences from
 * their sampled left and upper neighbours (tone: luma / (1 + luma) of the film's mean, 0 unless finite and positive),
 * -1 for a cell without samples; computed on the device, then set on the grid (x2_workgrid_set_scores). scores: each
 * cell's score (host array, may be null). The grid's size must be the film's. Waits. */
int x2_workgrid_score_film(x2_scene* scene, x2_workgrid* grid, float* scores);
/* The broker: its next launch's chunks, up to want, taken by its cellular workers (options.workers, seeded at the
 * first call), a share each, from their cells by the cellular rules. Returns how many. One broker thread a grid. */
uint32_t x2_workgrid_take(x2_workgrid* grid, uint32_t want, x2_chunk* out);
typedef struct x2_workgrid_result {
    uint64_t launches, chunks, samples;  /* wavefront launches made, chunks and samples rendered */
    float milliseconds;                  /* host time of the whole frame */
    float gpu_milliseconds;              /* the launches' device times, added */
} x2_workgrid_result;
/* A frame fed from a grid: the film cleared (x2_frame_begin), then launch after launch of up to chunks_per_launch
 * chunks (the broker's takes, x2_workgrid_take, until the launch is full or nothing more is handed out), each rendered
 * in the wavefront form and waited for, until the grid hands out nothing. The grid's size must be the scene's frame.
 * Waits. */
int x2_render_workgrid(x2_scene* scene, x2_workgrid* grid, uint32_t chunks_per_launch, x2_workgrid_result* result);

/* ---- differentiation (no reference counterpart; config 4) ----
 * The differentiable parameters, set in place: each material's diffuse colour (a Lambert lobe's albedo; 3 floats a
 * material), each material's roughness (a GGX lobe's; 1 float a material) and each light's radiance (3 floats a
 * light); host arrays, null leaves a set as it is. Waits. */
int x2_scene_set_params(x2_scene* scene, const float* albedo, const float* roughness, const float* radiance);
/* A texture's texels set in place (host array, the texture's width x height x 3 floats). Waits. */
int x2_scene_set_texture(x2_scene* scene, uint32_t texture, const float* rgb);
/* The adjoint of samples [first, first + count) of every pixel (the film's mean image): given dL/dimage (device, 3
 * floats a pixel), adds dL/dalbedo (device, 3 doubles a material: for a textured material its diffuse multiplier),
 * dL/droughness (device, 1 double a material; null: not wanted), dL/dradiance (device, 3 doubles a light) and
 * dL/dtexel (device, 3 doubles a texel over the scene's textures in order; null: not wanted; summed in FP32 before it
 * is added). Each sample's path is replayed from its identity (nothing
 * of a primal pass is stored) and each contribution credited to the light it reached and the Lambert and GGX vertices
 * it passed, the sampling decisions (directions, pdfs, MIS weights, roulette) held fixed. The replay runs in the
 * wavefront form (x2_wavefront_reserve paths in flight, x2_wavefront_tune's shape). Requires no volumes,
 * max_depth < 128, bsdf_samples = 1, 4 x materials + 3 x lights <= 24576. Waits. */
int x2_adjoint(x2_scene* scene, uint32_t first, uint32_t count, const float* d_dloss_dimage, double* d_albedo_grad,
               double* d_roughness_grad, double* d_radiance_grad, double* d_texture_grad);
/* x2_adjoint with its replay in the plain megakernel's form (one thread a sample) instead of the wavefront form: the
 * same estimator and results (up to the FP32 partial sums' order). */
int x2_adjoint_plain(x2_scene* scene, uint32_t first, uint32_t count, const float* d_dloss_dimage, double* d_albedo_grad,
                     double* d_roughness_grad, double* d_radiance_grad, double* d_texture_grad);
/* The last timed wavefront launch's queue sizes: for each iteration, rays extended then shadow rays (2 a
 * iteration, at most max values). */
int x2_wavefront_queues(x2_scene* scene, uint32_t* sizes, uint32_t max);
/* A wavefront launch that allocates nothing. No counterpart in the reference. For callers that cannot call
 * cudaMalloc: a process whose device memory another allocator already holds, or a path where cudaMalloc's implicit
 * device synchronisation is not allowed. Its scratch is one file-scope device array of at most 36 MiB that every GPU
 * loading the library holds until exit; the caller passes the chunks (device memory) and the film it adds to
 * (device: 4 doubles and one count a pixel; zero them first). Limits: at most 2^20 work items a call
 * (count x 64 x samples_per_chunk), light_count x light_samples <= 32, bsdf_samples = 1; beyond them X2_EINVAL.
 * Each chunk's count should be at most samples_per_chunk; a larger count renders samples_per_chunk samples of its
 * pixels (the chunks are in device memory and are not read on the host). Every call looks up the array's address
 * with the scene's device current, and the first call on a device loads the library's module there: make that first
 * call before any stream capture. Calls share the array: calls that overlap on the GPU race. Waits for the launch,
 * error returns included; after X2_ETIMEOUT wait for the scene's stream before the next call. *samples_done (or
 * null) gets the samples rendered. */
int x2_launch_wavefront_static(x2_scene* scene, const x2_chunk* d_chunks, uint32_t count, uint32_t samples_per_chunk,
                               double* d_sums, uint32_t* d_counts, uint64_t* samples_done);
int x2_film_download(x2_scene* scene, double* sums, double* odd, uint32_t* counts);  /* downloadFilm(); waits */
int x2_film_device(x2_scene* scene, double** d_sums, double** d_odd, uint32_t** d_counts);
int x2_audit(x2_scene* scene, const uint32_t* expected, int64_t* bad_pixel);  /* async_render.h:992-1048 */
int x2_counters_read(x2_scene* scene, x2_counters* out);  /* waits */
/* Measurement only (no reference counterpart): the device's cache read bandwidth in GB/s, the ceiling of the
 * traversal kernels' node and triangle fetches. level 2: a buffer of `bytes` (under the L2's size) swept `passes`
 * times by the whole grid; level 1: each block re-reading its own slice of min(bytes, 96 KiB). Allocates its buffer;
 * waits. */
int x2_probe_bandwidth(x2_ctx* ctx, uint32_t level, uint64_t bytes, uint32_t passes, float* gbs);
int x2_counters_reset(x2_scene* scene);
/* Counting mode (no reference counterpart; the algorithmic-bytes count of the roofline): launches made while it is
 * on count BVH node visits and triangle tests per ray. It slows them: never time a counting launch. */
int x2_count_traversal(x2_scene* scene, int on);
/* Each output is two counts: [0] closest-hit rays, [1] any-hit (shadow) rays. Waits; resets the counts. */
int x2_traversal_counts(x2_scene* scene, uint64_t* rays, uint64_t* nodes, uint64_t* triangles);
/* The wavefront traversal kernels' lane use in counting mode, six counts a ray kind ([0..5] closest hit, [6..11] any
 * hit): warp steps, live lanes summed over them, steps that visited a node, lanes that visited, triangle-test
 * iterations, lanes that tested. Waits; does not reset (x2_traversal_counts does). */
int x2_traversal_lanes(x2_scene* scene, uint64_t* lanes);

/* ---- host-side synthetic scenes (test and bench inputs, not the hot path) ----
 * config_id 0: the closed box with two boxes and a rect light; 1: heightfield + icospheres with 16 rect lights
 * and an environment; 100 + k: a config-1 variant scaled down by k (fewer tiles and spheres) for tests;
 * 200 + r (r < 48): batched request r (config-1-style, 0.1M..2M triangles, 128^2..1024^2, 4..256 spp, depth 4..32,
 * frame seed 1 + r); 300 + r: the same request shrunk (triangles / 64, resolution and spp / 8).
 * The descriptor and its arrays are owned by the library until x2_scene_desc_free. */
int x2_scene_generate(uint32_t config_id, uint64_t seed, x2_scene_desc** out, x2_config* config);
void x2_scene_desc_free(x2_scene_desc* desc);

#ifdef __cplusplus
}
#endif
#endif /* X2_H */
