/*
 * delta_ray_b200 -- C ABI of the B200-native differentiable edge-sampling path tracer.
 *
 * This is the drop-in replacement for the reference renderer's FFI: the
 * pybind11 module `delta_ray` (delta_ray.cpp:1838-1920) whose one compute entry
 * point is
 *     delta_ray.render(Camera, [Shape], [Material], [Light], (W, H), d_image,
 *                      num_samples, max_bounces, seed, print_progress)
 *         -> RenderResult                                  (delta_ray.cpp:1017)
 * The reference decides forward vs backward by the rank of d_image
 * (delta_ray.cpp:1029); here they are two entry points.  The reference builds
 * its scene on every call (delta_ray.cpp:1030); here the scene is built once by
 * dr_scene_create and reused, and dr_scene_update refreshes vertex positions.
 *
 * Conventions
 *  - Plain C types only; every pointer inside a descriptor may be host or
 *    device memory (CUDA unified addressing tells them apart) unless stated.
 *  - Matrices are 4x4 row-major float32, exactly the reference's numpy layout.
 *  - All calls are stream-ordered on the given cudaStream_t (passed as void*,
 *    NULL = legacy default stream).  Image and gradient outputs are device
 *    pointers.  A scene must not be used by two calls concurrently.
 *  - Every call returns a dr_status; on failure dr_last_error() describes it.
 *    Device-side failures are reported through a status word, never a trap.
 */
#ifndef DELTA_RAY_B200_H
#define DELTA_RAY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DR_ABI_VERSION 2

#if defined(__GNUC__)
#define DR_API __attribute__((visibility("default")))
#else
#define DR_API
#endif

typedef enum {
    DR_OK = 0,
    DR_ERR_INVALID_ARGUMENT = 1,
    DR_ERR_CUDA = 2,
    DR_ERR_OUT_OF_MEMORY = 3,
    DR_ERR_DEVICE_STATUS = 4, /* a kernel reported an error word (bounds, queue overflow) */
    DR_ERR_NOT_SUPPORTED = 5
} dr_status;

/* Camera (camera.h:12-22 of the reference).  fov_factor = tan(fov / 2),
 * aspect_ratio = width / height.  Only cam_to_world, fov_factor and
 * aspect_ratio shape the camera rays (camera.h:49-84); world_to_cam and
 * clip_near shape edge projection (camera.h:218-242). */
typedef struct {
    const float *cam_to_world;  /* [16] */
    const float *world_to_cam;  /* [16] */
    const float *sample_to_cam; /* [16] */
    const float *cam_to_sample; /* [16] */
    float fov_factor;
    float aspect_ratio;
    float clip_near;
    int fisheye;
} dr_camera_desc;

/* Material (material.h:14-22).  A channel with tex_w == tex_h == 0 is a
 * constant ([3] or [1]); otherwise it is a [tex_h][tex_w][c] texture with
 * bilinear wrap-around lookup (material.h:108-203). */
typedef struct {
    const float *diffuse;   /* [3] or [h][w][3] */
    int diffuse_w, diffuse_h;
    const float *specular;  /* [3] or [h][w][3] */
    int specular_w, specular_h;
    const float *roughness; /* [1] or [h][w][1] */
    int roughness_w, roughness_h;
    const float *diffuse_uv_scale;   /* [2] */
    const float *specular_uv_scale;  /* [2] */
    const float *roughness_uv_scale; /* [2] */
    int two_sided;
    /* Specular lobe: DR_MICROFACET_BLINN_PHONG (the reference's, material.h:
     * 257-462) or DR_MICROFACET_GGX (Walter et al. 2007: alpha = roughness^2,
     * exact Smith G1; no counterpart in the reference). */
    int microfacet;
} dr_material_desc;

typedef enum { DR_MICROFACET_BLINN_PHONG = 0, DR_MICROFACET_GGX = 1 } dr_microfacet;

/* Triangle mesh (shape.h:11-18). */
typedef struct {
    const float *vertices; /* [num_vertices][3] */
    int num_vertices;
    const int *indices;    /* [num_triangles][3] */
    int num_triangles;
    const float *uvs;      /* [num_vertices][2] or NULL */
    const float *normals;  /* [num_vertices][3] or NULL (shading normals) */
    int material_id;
} dr_shape_desc;

/* Area light (light.h:15-18): every triangle of shape_id emits intensity. */
typedef struct {
    int shape_id;
    const float *intensity; /* [3] */
} dr_light_desc;

typedef struct {
    dr_camera_desc camera;
    const dr_material_desc *materials;
    int num_materials;
    const dr_shape_desc *shapes;
    int num_shapes;
    const dr_light_desc *lights;
    int num_lights;
    /* Optional LTC tables for edge sampling of Blinn-Phong and GGX lobes,
     * 128*128 row-major 3x3 float32 matrices indexed [roughness_bin +
     * theta_bin * 128] (ltc.inc:2-4, material.h:464-476).  NULL selects
     * identity matrices (edges sampled by the cosine lobe, unbiased); the
     * Python layer passes the fitted tables of delta_ray_b200/data. */
    const float *ltc_table;
    const float *ltc_table_ggx;
} dr_scene_desc;

/* How the per-secondary-point edge position derivative is pushed back
 * through the path (delta_ray.cpp:976-1002).  The reference *sets* the
 * adjoint once per edge, so only the last edge of each shading point
 * survives; DR_DP_SUM adds every edge (the unbiased estimator). */
typedef enum { DR_DP_REFERENCE_LAST = 0, DR_DP_SUM = 1 } dr_dp_mode;

/* dr_render_desc.flags.  DR_FLAG_FULL_PIXEL_JITTER spreads each pixel's
 * samples over the whole pixel (a box filter).  Without it the sub-pixel
 * offset is u / spp in each axis, as in the reference (delta_ray.cpp:1236-1237),
 * so that all samples of a pixel fall in its [0, 1/spp)^2 corner: the image is
 * then nearly point-sampled, while the primary-edge gradient is the derivative
 * of the box-filtered image.  DR_FLAG_DETACHED_PDF holds the BSDF sampling
 * pdf constant in the backward pass.  The reference differentiates it while
 * keeping the sampled direction fixed (pathtrace.h:248-253), which biases the
 * gradient of every parameter that shapes the sampling (roughness, the lobe
 * weights) by -E[contribution * d log pdf]; held constant it is unbiased.
 * DR_FLAG_EDGE_LOBE_MIS changes the weight of a secondary-edge sample.
 * The reference picks one lobe (diffuse or specular) with probability pmf,
 * samples the edge by that lobe's line pdf, and divides the sample by
 * pmf * line pdf (delta_ray.cpp:88-105, 318-330). The sample evaluates the whole
 * BSDF, so the expectation is the edge integral once per lobe with nonzero pmf,
 * twice the integral on materials with both lobes. With the flag the sample is
 * divided by the mixture density, the sum over both lobes of pmf * that lobe's
 * line pdf at the sampled point (the one-sample balance heuristic). That is
 * unbiased wherever either lobe can sample the edge.
 * DR_FLAG_LEARNED_PROPOSAL draws secondary edges with the scene's learned
 * proposal (dr_scene_set_proposal) and, in its training mode, takes one
 * training step per backward call; see dr_proposal_desc. */
typedef enum {
    DR_FLAG_FULL_PIXEL_JITTER = 1,
    DR_FLAG_DETACHED_PDF = 2,
    DR_FLAG_EDGE_LOBE_MIS = 4,
    DR_FLAG_LEARNED_PROPOSAL = 8
} dr_render_flags;

typedef struct {
    int width;
    int height;
    int spp;          /* samples per pixel (num_samples) */
    int max_bounces;
    uint64_t seed;
    /* Number of primary-edge samples in the backward pass; <= 0 selects
     * spp * width * height, the reference's total over all its threads
     * (delta_ray.cpp:1474-1475 with one thread). */
    int64_t primary_edge_samples;
    int dp_mode;      /* dr_dp_mode */
    int flags;        /* dr_render_flags */
    int reserved[7];  /* must be zero */
} dr_render_desc;

/* Gradient layout: one flat float32 buffer, in this order
 *   d_cam_to_world[16] d_world_to_cam[16] d_sample_to_cam[16] d_cam_to_sample[16]
 *   for each material: d_diffuse (3 or h*w*3), d_specular (3 or h*w*3),
 *                      d_roughness (1 or h*w)
 *   for each shape:    d_vertices (3V), then d_normals (3V) when the shape has normals
 *   for each light:    d_intensity (3)
 * (the fields of RenderResult / DCamera / DMaterial / DShape / DLight,
 * delta_ray.cpp:1007-1015).  dr_scene_grad_layout reports the offsets. */
typedef struct {
    size_t total;                 /* floats in the flat buffer */
    size_t camera;                /* offset of d_cam_to_world; the other 3 follow */
    const size_t *material;       /* [num_materials * 3]: diffuse, specular, roughness */
    const size_t *shape_vertices; /* [num_shapes] */
    const size_t *shape_normals;  /* [num_shapes], (size_t)-1 when absent */
    const size_t *light;          /* [num_lights] */
} dr_grad_layout;

typedef struct dr_scene dr_scene;

/* Library/ABI version; lets a binding check what it loaded. */
DR_API int dr_abi_version(void);

/* Builds the device scene: geometry, LBVH, light samplers, edge list,
 * primary-edge sampler and edge trees (scene.cpp:19-136). */
DR_API dr_status dr_scene_create(const dr_scene_desc *desc, int device, dr_scene **out);

/* Replaces vertex positions (same topology) and rebuilds what depends on
 * them; `desc` must describe the same meshes as at creation. */
DR_API dr_status dr_scene_update(dr_scene *scene, const dr_scene_desc *desc);

DR_API dr_status dr_scene_destroy(dr_scene *scene);

DR_API dr_status dr_scene_grad_layout(const dr_scene *scene, dr_grad_layout *layout);

/* Forward render: image [H][W][3] float32 (device), the mean over spp
 * samples of each pixel (delta_ray.cpp:1190-1333, render_sample_fast
 * :640-692).  Overwrites the image. */
DR_API dr_status dr_render_forward(dr_scene *scene, const dr_render_desc *rd, float *image_dev,
                            void *stream);

/* Backward render (delta_ray.cpp:694-1005 and :1468-1550): given the image
 * adjoint d_image [H][W][3] (device), overwrites grad_dev (device, flat
 * layout above) with every parameter gradient.  image_dev may be NULL;
 * otherwise the re-rendered image is written there too.  Paths are
 * differentiated through "specular" samples (roughness <= 0.01), and the
 * vertices such samples reach are shading points too (pathtrace.h:141-227);
 * a path keeps at most 8 such vertices differentiable.  The library's item
 * queue holds up to 8 GiB of sampled edges; larger edge stages (glossy
 * scenes with many edges sample thousands per shading point) are evaluated
 * in several passes over the shading points. */
DR_API dr_status dr_render_backward(dr_scene *scene, const dr_render_desc *rd, const float *d_image_dev,
                             float *grad_dev, float *image_dev, void *stream);

/* One view of a multi-view backward render: a camera (the layout of
 * dr_scene_desc.camera), its render settings and its image adjoint
 * (d_image [render.height][render.width][3], device); image (device, may be
 * NULL) receives the view's re-rendered image. */
typedef struct {
    dr_camera_desc camera;
    dr_render_desc render;
    const float *d_image;
    float *image;
} dr_view_desc;

/* Backward render of several views of the scene in one call (no counterpart
 * in the reference, which renders one camera per call): each view is rendered
 * with its own camera, resolution, samples, bounces and seed on the
 * library's queues, and its primary edges are sampled from its own camera.
 * grad_dev (flat layout) receives the sum over the views of every
 * non-camera gradient, with its camera block zero; camera_grads_dev
 * ([n_views][64] floats, device, may be NULL) receives each view's camera
 * gradient (cam_to_world, world_to_cam, sample_to_cam, cam_to_sample).
 * Returns after the stream has finished. */
DR_API dr_status dr_render_backward_views(dr_scene *scene, int n_views, const dr_view_desc *views, float *grad_dev,
                                          float *camera_grads_dev, void *stream);

/* Backward render that allocates no device memory.  No counterpart in the
 * reference (whose backward allocates per call, delta_ray.cpp:1468-1550): it
 * serves callers that must not allocate during a render, e.g. a process whose
 * device memory is all reserved by its own pool.  Same computation and
 * arguments as dr_render_backward, but its work queues live in a fixed 32 MiB
 * array per device that is part of the library's module image.  Limits:
 * width * height * spp <= 65536 (larger calls fail with
 * DR_ERR_INVALID_ARGUMENT); sampled edges beyond the array's room (about
 * 330,000 at the largest image) are evaluated in several passes over the
 * shading points, and a single point with more edges than that fails with
 * DR_ERR_OUT_OF_MEMORY, as do specular chains whose shading points outgrow
 * half the array (about 150,000 points).  All calls on
 * one device share the array, so overlapping calls (from several threads or
 * streams) race: serialize them.  Where CUDA loads modules and kernels
 * lazily, the array's memory and the kernels' code are taken when a scene is
 * created on the device (dr_scene_create looks the array up and loads every
 * kernel a backward call launches), not by this call; each call looks up the
 * address of the current context's copy again. */
DR_API dr_status dr_render_backward_noalloc(dr_scene *scene, const dr_render_desc *rd, const float *d_image_dev,
                                            float *grad_dev, float *image_dev, void *stream);

/* Upper bound on the edge items a dr_render_backward call holds on the
 * device at once (64 bytes each); 0 restores the default, 8 GiB worth
 * (134,217,728 items).  A call whose shading points sample more edges runs its
 * edge stage in chunks of points whose edges fit, planned from the edge
 * counts of a full pass or of the previous call on the same scene; the
 * results do not depend on the bound.  Process-wide; a negative bound fails
 * with DR_ERR_INVALID_ARGUMENT.  No counterpart in the reference, whose CPU
 * renderer evaluates each edge as it samples it. */
DR_API dr_status dr_set_item_queue_limit(int64_t items);

/* A scene's queue settings for its backward calls (no counterpart in the
 * reference, whose CPU renderer has no work queues).  Large edge trees are
 * walked in two stages: each point's walk down to 8 levels below the roots,
 * then the subtrees there.
 *   depth_first: 0 (the default) walks those subtrees level by level, one
 *     launch per level over every subtree's nodes of that level; 1 walks
 *     each subtree depth first, one lane per subtree;
 *   hand_steps: with depth_first, the node steps a subtree walk takes before
 *     it hands its shallowest pending subtree on to the next round
 *     (1..4096; default 64);
 *   task_rounds: with depth_first, launches of the subtree stage per chunk of
 *     shading points, the last handing nothing on (1..8; default 3);
 *   queue_items: bound on the edge items the scene's calls hold at once (0,
 *     the default: the process-wide bound of dr_set_item_queue_limit; else
 *     the smaller of the two);
 *   reserved: 0.
 * No setting changes which edges are sampled or what they contribute: the
 * counts and the image are the same under every setting, the gradient up to
 * float round-off (atomic adds sum in another order). */
typedef struct {
    int32_t hand_steps;
    int32_t task_rounds;
    int64_t queue_items;
    int32_t depth_first;
    int32_t reserved;
} dr_tuning;

DR_API dr_status dr_scene_get_tuning(const dr_scene *scene, dr_tuning *out);
/* Out-of-range values fail with DR_ERR_INVALID_ARGUMENT. */
DR_API dr_status dr_scene_set_tuning(dr_scene *scene, const dr_tuning *tuning);

/* What dr_scene_autotune measured: the setting it chose, its time per
 * backward call, the time of the setting the scene had before (ms, host wall
 * time to the end of the call's stream work) and the settings it timed. */
typedef struct {
    dr_tuning best;
    float best_ms;
    float start_ms;
    int32_t trials;
} dr_tune_report;

/* Chooses the scene's queue settings by timing backward calls of this render
 * (arguments as dr_render_backward; grad_dev holds the last call's gradient
 * afterwards).  Coordinate search from the current setting: the subtree walk,
 * and for the depth-first one its rounds 1-4 and hand-on steps 16-256 (only
 * where points hand subtrees on), then
 * item-queue bounds of 1/2, 1/4 and 1/8 of the last call's items (smaller
 * chunks of the edge stage, whose queues sit nearer to L2); each setting
 * timed as the faster of two calls, at most max_trials settings.  The fastest
 * stays set on the scene, so calls of the same kind (an inverse-rendering
 * loop) can be tuned once, before the loop.  report may be NULL.  On failure
 * the scene keeps the setting it had. */
DR_API dr_status dr_scene_autotune(dr_scene *scene, const dr_render_desc *rd, const float *d_image_dev,
                                   float *grad_dev, int max_trials, dr_tune_report *report, void *stream);

/* Closest hits of n rays [n][6] (origin, direction; device memory) on
 * (1e-3, inf): global triangle id (-1 on a miss; ids run over shapes in
 * order, then triangles) and distance.  Replaces the reference's
 * nearest_hit (scene.cpp:177-202) and uses the same hit rule as the
 * renderer's own traversal. */
DR_API dr_status dr_trace_rays(dr_scene *scene, const float *rays_dev, int64_t n, int *tri_dev, float *t_dev,
                        void *stream);

/* Check hook (no counterpart in the reference, whose transcendental functions
 * are the host libm's): evaluates the renderer's reproducible float functions
 * on the device, out[i] = f(x[i]) or f(x[i], y[i]) for fn 0 sin, 1 cos,
 * 2 atan, 3 atan2(x, y), 4 acos, 5 exp, 6 log, 7 pow(x, y) (device buffers of
 * n floats; y may be NULL except for atan2 and pow).  The same functions,
 * compiled for the host, give the same bits; tests compare the two.  Returns
 * after the stream has finished. */
DR_API dr_status dr_eval_math(int fn, const float *x_dev, const float *y_dev, float *out_dev, int64_t n,
                              void *stream);

/* Tooling: per-stage GPU time of the following render calls.  With
 * profiling on, each render records CUDA events around its kernels and
 * synchronizes its stream at the end; dr_scene_last_timings then returns
 * stage `index` (name and milliseconds) of the last call, DR_ERR_INVALID_ARGUMENT
 * past the last stage.  No counterpart in the reference (its only timer is the
 * progress reporter, progress_reporter.h:7-47). */
DR_API dr_status dr_scene_set_profiling(dr_scene *scene, int enable);
DR_API dr_status dr_scene_last_timings(const dr_scene *scene, int index, char *name, size_t name_len, float *ms);

/* Work counts of the last backward call: secondary shading points and
 * sampled edges (tooling). */
DR_API dr_status dr_scene_last_counts(const dr_scene *scene, int64_t *points, int64_t *items);

/* Tooling: one array of the scene's edge data, as built (no counterpart in
 * the reference, whose edge trees live in its Scene, scene.cpp:91-97):
 * what 0 silhouette-tree nodes (56 B each: box, cone axis and angle, offset,
 * edge count, total length, pad), 1 silhouette-tree edges in leaf order
 * (20 B: shape, v0, v1, f0, f1), 2 normal-tree nodes, 3 normal-tree edges,
 * 4 primary edges, 5 primary cdf (float), 6 primary func (float), 7 the
 * primary func integral (one float).  *count receives the element count; up
 * to capacity_bytes are copied to out_host (may be NULL).  build_ms (may be
 * NULL) receives the host wall time of the scene's last GPU edge build (0 for
 * scenes of at most 8192 triangles, which build on the host). */
DR_API dr_status dr_scene_edge_data(const dr_scene *scene, int what, void *out_host, int64_t capacity_bytes,
                                    int64_t *count, float *build_ms);

/* Tooling: work counts of the last backward call (the inputs of a byte model
 * of its kernels; no counterpart in the reference): counts[0] shading points,
 * [1] sampled edges, [2] line samples kept for their rays (in scenes
 * traced through the LBVH: those whose rays hit one of the edge's faces),
 * [3] samples kept for shading, [4] subtrees walked by the second traversal
 * stage (handed on by the first stage, and with the depth-first walk between
 * its rounds),
 * [5] edges sampled by the first stage (all, when the traversal runs in one
 * stage), [6] edge-tree nodes visited by the point walks, [7] nodes
 * visited by the subtree walks, [8] line samples whose connectivity test
 * passed (candidates of the ray stage), [9] subtrees the level walk left to
 * a lane's depth-first walk because a level's queue was full.  Up to n of
 * them are written. */
DR_API dr_status dr_scene_last_work(const dr_scene *scene, int64_t *counts, int n);

/* Kernel launch count of the last render call on this scene (for tooling). */
DR_API dr_status dr_scene_last_launch_count(const dr_scene *scene, int *count);

/* Copies the last error message of the calling thread into buf. */
DR_API size_t dr_last_error(char *buf, size_t len);

/* The learned edge proposal's network (no counterpart in the reference): a
 * 10 -> 64 -> 64 -> 64 -> 32 MLP (ReLU, softmax output) run on the tensor
 * cores in bf16 with f32 accumulation.  params: dr_mlp_param_count() floats
 * (device), W1 [64][16] (the proposal fills 10 inputs and zeroes 10..15), b1 [64], W2 [64][64],
 * b2, W3 [64][64], b3, W4 [32][64], b4 [32]; weight[out][in] row-major.
 * x: [n][16] f32 rows (device), rounded to bf16 as the kernels read them.
 * dr_mlp_forward writes the logits [n][32].  dr_mlp_gradient overwrites
 * grads with the gradient of  sum_rows sum_s -t[s] log softmax(z)[s] / T  (T
 * the sum of all targets) and *loss with that loss.  Both synchronize the
 * stream; they allocate their own scratch. */
DR_API int dr_mlp_param_count(void);

/* The learned edge proposal of a scene (no counterpart in the reference,
 * which samples edges by the edge trees' importance alone).  With
 * DR_FLAG_LEARNED_PROPOSAL a backward call computes, for every shading point,
 * the network's probabilities over 32 directions from the point (4 bands of
 * cos(theta) times 8 azimuth sectors in the shading frame) from the point's
 * position (normalised to the scene bounds), shading normal, roughness and
 * incoming direction.  With probability `mix` the edge trees' all-mode
 * traversal then picks children in proportion to their importance times the
 * probability of the direction towards them, and by importance alone
 * otherwise: a defensive mixture whose exact pmf enters the reference's
 * multiple-importance weights, so the gradient stays unbiased for any
 * network.  In training mode each such call sums the contribution magnitude
 * |dv0| + |dv1| of every sampled edge per direction of its midpoint for
 * `train_points` shading points spread over the call's points and takes one
 * Adam step on  sum -t log q / sum t  (t the magnitudes, q the network's
 * probabilities). */
typedef struct {
    int train;             /* 1: one training step per backward call that uses the proposal */
    float mix;             /* probability of the learned descent, in [0, 1] */
    float learning_rate;   /* Adam step size */
    int64_t train_points;  /* shading points per training step (<= 0: 32768) */
    const float *params;   /* dr_mlp_param_count() floats, host or device; NULL keeps the
                              current parameters (a fixed initialisation the first time) */
} dr_proposal_desc;
DR_API dr_status dr_scene_set_proposal(dr_scene *scene, const dr_proposal_desc *desc);
/* Current parameters (params_out: host or device, may be NULL), the last
 * training loss and the number of training steps taken. */
DR_API dr_status dr_scene_proposal_state(const dr_scene *scene, float *params_out, float *last_loss, int64_t *steps);
DR_API dr_status dr_mlp_forward(const float *params_dev, const float *x_dev, int64_t n, float *logits_dev,
                                void *stream);
DR_API dr_status dr_mlp_gradient(const float *params_dev, const float *x_dev, const float *targets_dev, int64_t n,
                                 float *grads_dev, float *loss_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DELTA_RAY_B200_H */
