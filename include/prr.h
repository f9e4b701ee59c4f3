/*
 * prr.h -- C ABI of libprr, the B200 (sm_100a) Monte Carlo path-tracing hot
 * path of the PhotoRealisticRender4610 CPU renderer.
 *
 * The reference has no plugin or FFI layer: its interface is a set of C++
 * classes compiled into one executable (Scene, BVHAccel, Integrator, Renderer,
 * tonemap). Each entry point below names the reference member it replaces
 * (file:line in the reference tree). The C++ drop-in classes in prr_dropin.hpp
 * forward to these calls with the reference's own class and method names.
 *
 * Conventions
 *   - Every call returns an int status: PRR_OK (0) or a negative PRR_ERR_*;
 *     prr_last_error() gives the calling thread's message for the last failure.
 *   - Handles are opaque. A scene is immutable after prr_scene_build() and may
 *     then be used from several host threads and streams at once.
 *   - Unless a name ends in _host, array arguments are DEVICE pointers owned by
 *     the caller and the call is asynchronous on `stream` (a cudaStream_t, NULL
 *     for the legacy default stream). _host variants take host pointers and
 *     return when the results are in host memory.
 *   - Rays are n x 3 float arrays of origins and of directions (x,y,z per ray).
 */
#ifndef PRR_H
#define PRR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PRR_ABI_VERSION 1

#define PRR_OK 0
#define PRR_ERR_INVALID_ARGUMENT (-1)
#define PRR_ERR_CUDA (-2)
#define PRR_ERR_OUT_OF_MEMORY (-3) /* a device (or pinned host) allocation failed */
#define PRR_ERR_NOT_BUILT (-4)
#define PRR_ERR_UNSUPPORTED (-5)
#define PRR_ERR_TIMEOUT (-6)
#define PRR_ERR_BUDGET (-7)
#define PRR_ERR_INTERNAL (-8)

/* Material kinds: DiffuseMaterial, EmissiveMaterial, MirrorMaterial,
 * GlassMaterial (Material.hpp:120-183). */
#define PRR_MAT_DIFFUSE 0
#define PRR_MAT_EMISSIVE 1
#define PRR_MAT_MIRROR 2
#define PRR_MAT_GLASS 3

/* MaterialType of GLTFLoader::load (GLTFLoader.hpp:10) */
#define PRR_GLTF_DIFFUSE 0
#define PRR_GLTF_GLASS 1
#define PRR_GLTF_MIRROR 2
#define PRR_GLTF_EMIT 3

typedef struct prr_scene prr_scene;
typedef struct prr_photon_map prr_photon_map;

/* Tone mappers: tonemap::ToneMapper (ToneMapping.hpp:32-37) plus ACES. */
#define PRR_TONEMAP_RAW 0
#define PRR_TONEMAP_STANDARD 1
#define PRR_TONEMAP_AGX 2
#define PRR_TONEMAP_PBR_NEUTRAL 3
#define PRR_TONEMAP_ACES 4 /* new: K. Narkowicz's ACES filmic fit + sRGB OETF */

/* Camera fields of Camera::create + aperture/focusDistance (Camera.hpp:10-31). */
typedef struct prr_camera {
    float eye[3], target[3], up[3];
    float fovv, fovh;
    float aperture;
    float focus_distance; /* < 0: distance eye -> target (Camera.hpp:51-54) */
} prr_camera;

/* Traversal launch shape (chosen by the autotuner; zero fields = defaults). */
typedef struct prr_trace_config {
    int block_size;   /* threads per block (multiple of 32) */
    int persistent;   /* 0: one ray per thread; 1: persistent grid, each warp
                         takes 32 rays at a time; 2: persistent grid, lanes whose
                         ray finished take new rays as soon as `batch` lanes of the
                         warp are idle; 3: as 2, with postponed leaves (node and
                         triangle steps in separate warp-wide phases) */
    int blocks_per_sm;/* persistent grids: resident blocks per SM (0 = occupancy) */
    int batch;        /* modes 2-3: refill threshold in idle lanes (0 = 8) */
    int leaf_batch;   /* mode 3: a triangle phase runs when this many lanes hold a
                         parked leaf (0 = 16) */
    int sort_rays;    /* 0: trace rays in input order; 1-5: first reorder them by a
                         coherence key so neighbouring lanes trace similar rays: where
                         each ray enters the mesh's root box and its direction,
                         interleaved (1), direction-major (2) or entry-major (3); or
                         where it enters and where it leaves the box, interleaved (4)
                         or entry-major (5).
                         Results are written at each ray's input index either way
                         and do not depend on the order. Batches of 2^31 rays or
                         more are traced in input order. */
} prr_trace_config;

#define PRR_RENDER_PLAIN 0     /* one megakernel thread per (pixel, sample range) */
#define PRR_RENDER_WAVEFRONT 1 /* staged wavefront integrator */

/* RenderSettings (Renderer.hpp:42-55) plus the integrator's knobs. */
typedef struct prr_render_settings {
    int width, height;        /* must equal the camera's (Camera::init) */
    int min_spp, max_spp;     /* minSPP == maxSPP: fixed spp; else the Welford
                                 confidence stop of Renderer.cpp:88-95 */
    int max_depth;            /* Integrator maxDepth */
    float variance_threshold; /* varianceThreshold */
    float indirect_clamp;     /* Integrator::indirectClamp (10 in the reference) */
    int mode;                 /* PRR_RENDER_PLAIN / PRR_RENDER_WAVEFRONT */
    uint64_t seed;            /* sample n of pixel m = i + j*W draws stream (seed, m, n) */
    int x0, y0, x1, y1;       /* pixel window [x0,x1) x [y0,y1); x1 or y1 <= 0: full frame */
    int sample_offset;        /* index of the first sample (progressive passes, resume) */
    int slices;               /* plain fixed-spp mode: threads per pixel (0 = automatic) */
} prr_render_settings;

/* Wavefront launch shape (chosen by prr_autotune; zero fields = defaults). */
typedef struct prr_wavefront_config {
    int64_t paths_per_pass; /* paths in flight per pass (0: about 8M; at most 2^30; about
                               320 bytes of device memory each) */
    int block_size;         /* threads per block of the traversal stages (0: 128) */
    int use_graphs;         /* 1: replay each pass from one captured CUDA graph */
    int stack_smem;         /* mesh-BVH stack entries per thread kept in shared memory;
                               deeper entries spill to a global buffer (0: the whole stack) */
    int ordered;            /* 1: rebuild the stage queues in path order (stable partition,
                               next rays grouped by direction octant); 0: append order */
    int refill;             /* traversal stages: a warp takes new rays from its queue once
                               this many of its lanes are idle (0: 8; at most 32) */
} prr_wavefront_config;

typedef struct prr_scene_stats {
    int64_t n_objects, n_triangles, n_nodes;
    int32_t tlas_depth, blas_depth;
    int64_t device_bytes;
    float total_emit_area;
    int64_t last_render_launches; /* kernels launched by the last prr_render on this scene */
} prr_scene_stats;

/* ---- library ---------------------------------------------------------- */
int prr_abi_version(void);
/* Copies the calling thread's last error message (NUL-terminated). Returns
 * its full length. */
int prr_last_error(char *buf, size_t len);

/* ---- BVH construction alone (BVHAccel ctor, BVH.cpp:13-54) --------------
 * Host-only: builds the reference's binned-SAH tree over n primitives given
 * their bounds (n x 6: minX,minY,minZ,maxX,maxY,maxZ) and areas, with
 * maxPrimsInNode clamped to 255, and writes the flattened layout (BVHNode
 * bounds interleaved per axis, first_child, meta, nodeAreas, orderedPrims).
 * Outputs must hold 2n-1 nodes; any may be NULL. Returns the node count. */
int64_t prr_bvh_build(const float *prim_bounds, const float *prim_areas, int64_t n,
                      int max_prims_in_node, float *bounds, uint32_t *first_child,
                      uint32_t *meta, float *areas, int32_t *ordered, int32_t *max_depth);

/* ---- scene (Scene, Scene.hpp:15-41) ------------------------------------ */
int prr_scene_create(prr_scene **out);
int prr_scene_destroy(prr_scene *scene);
/* params: baseColor[3], roughness, metallic, ior, emission[3]
 * (Material fields, Material.hpp:40-44). */
int prr_scene_add_material(prr_scene *scene, int kind, const float params[9], int *out_id);
/* MeshTriangle(tris, bounds, mat) (Triangle.hpp:116-124) + Scene::Add:
 * verts = ntri x 9 host floats (v0, v1, v2). The mesh gets its own BVH with
 * maxPrimsInNode 4 (Triangle.hpp:173-179). */
int prr_scene_add_mesh(prr_scene *scene, const float *verts, int64_t ntri, int material,
                       int *out_object);
/* MeshTriangle from triangles with per-corner data (Triangle.hpp:17-23), the
 * fields as a Triangle holds them: normals = ntri x 9 (n0, n1, n2, used as
 * given -- the glTF loader normalizes them first, GLTFLoader.cpp:237-239 -- and
 * the face normal becomes normalize(n0 + n1 + n2)), uvs = ntri x 6 (t0, t1,
 * t2), tangents = ntri x 12 (xyz + handedness w per corner). Any of the three
 * may be NULL. Hits on the mesh interpolate them as Triangle::finalize does
 * (Triangle.cpp:34-59). */
int prr_scene_add_mesh_attr(prr_scene *scene, const float *verts, const float *normals,
                            const float *uvs, const float *tangents, int64_t ntri, int material,
                            int *out_object);
/* A material texture (Texture, TextureUtils.hpp:9-18): width x height texels
 * of 3 or 4 8-bit channels, row-major, as decoded from the image file. */
int prr_scene_add_texture(prr_scene *scene, const uint8_t *texels, int width, int height,
                          int channels, int *out_texture);
/* Material::baseColorTex / metallicRoughnessTex / normalTex / emissiveTex
 * (Material.hpp:45-48): texture ids from prr_scene_add_texture, -1 for none.
 * Sampled bilinearly with wrap-around (TextureUtils.hpp:22-136) when shading
 * data is built (Material.cpp:3-26). */
int prr_scene_set_material_textures(prr_scene *scene, int material, int base_color,
                                    int metallic_roughness, int normal, int emissive);
/* GLTFLoader::load(path, type, override) + Scene::Add of every mesh it returns
 * (GLTFLoader.cpp:140-281): a .glb, or a .gltf with external or base64
 * buffers; one mesh per triangle primitive with its per-corner normals, uvs and
 * tangents; a new material per primitive from the glTF material recast to
 * `material_type` (PRR_GLTF_*), or `override_material` (>= 0) for all; PNG
 * textures decoded to 8-bit RGBA. Node transforms are not applied (the
 * reference reads primitives in mesh space). out_first / out_count: the objects
 * added; out_undecoded: images left out (JPEG, interlaced PNG). Primitives
 * without triangles add nothing. */
int prr_scene_add_gltf(prr_scene *scene, const char *path, int material_type,
                       int override_material, int *out_first, int *out_count, int *out_undecoded);
/* MeshTriangle(filename, offset, m) + Scene::Add (Triangle.cpp:4-32): the
 * first mesh of an OBJ file read as the reference's bundled loader reads it
 * (OBJ_Loader.hpp LoadFile), its face corners taken three at a time as
 * triangles, positions + offset (NULL: none). The file must end in ".obj" and
 * hold exactly one mesh (the reference asserts it), with a corner count that
 * is a multiple of three. */
int prr_scene_add_obj(prr_scene *scene, const char *path, const float *offset, int material,
                      int *out_object);
/* The triangles prr_scene_add_obj would add (ntri x 9 floats): with out_verts
 * NULL only *out_ntri is set; else out_verts holds `capacity` triangles. */
int prr_obj_read(const char *path, const float *offset, float *out_verts, int64_t capacity,
                 int64_t *out_ntri);
/* Host-side view of a mesh as added (before or after the build): ntri, the
 * kinds of per-corner data it carries (1 normals, 2 uvs, 4 tangents), and, for
 * non-NULL arrays, its triangles (ntri x 9), corner normals (ntri x 9), uvs
 * (ntri x 6) and tangents (ntri x 12), in input order. */
int prr_scene_export_mesh(const prr_scene *scene, int object, int64_t *out_ntri, int *out_attr,
                          float *verts, float *normals, float *uvs, float *tangents);
/* A material as added: kind, params[9] and its four texture ids (-1 none). */
int prr_scene_export_material(const prr_scene *scene, int material, int *out_kind,
                              float params[9], int textures[4]);
/* A texture as added: size, channels and (texels non-NULL) its texels. */
int prr_scene_export_texture(const prr_scene *scene, int texture, int *out_width,
                             int *out_height, int *out_channels, uint8_t *texels);
/* Sphere(center, radius, mat) (Sphere.hpp:14-16) + Scene::Add. */
int prr_scene_add_sphere(prr_scene *scene, const float center[3], float radius, int material,
                         int *out_object);
/* Scene::backgroundColor (Scene.hpp:17). */
int prr_scene_set_background(prr_scene *scene, const float rgb[3]);
/* EnvMap pixels (EnvMap.hpp:35-56 after decoding): w*h*3 host floats. */
int prr_scene_set_env(prr_scene *scene, const float *rgb, int width, int height);
/* Camera::init(width, height) (Camera.hpp:43-56). */
int prr_scene_set_camera(prr_scene *scene, const prr_camera *camera, int width, int height);
/* Scene::buildBVH (Scene.cpp:15-27): per-mesh SAH BVHs, the scene BVH over
 * objects (maxPrimsInNode 1), the emitter list, the env-map CDF (built on the
 * device, EnvMap.hpp:189-224), and the upload of everything. */
int prr_scene_build(prr_scene *scene, void *stream);
int prr_scene_stats_get(const prr_scene *scene, prr_scene_stats *out);
/* The device-side checks of the checked build (libprr_checked.so, compiled
 * with -DPRR_CHECKED), no counterpart in the reference: every node and
 * triangle fetch of the traversal kernels is tested against the array's
 * length, every stack push against its column's depth (the tree depth + 1),
 * every wavefront queue length and append against the queue's capacity. A
 * failed test keeps the access in bounds and records out[0] = the first error
 * (1 node index, 2 triangle index, 3 stack depth, 4 queue slot or length),
 * out[1] = its offending value, out[2] = the number of failed tests, in the
 * scene's status words. Waits for the device; reset != 0 clears the words.
 * Returns 1 in the checked build, 0 in the normal one (whose words stay 0). */
int prr_check_status(prr_scene *scene, uint32_t out[3], int reset);
/* The reference-layout flattened tree of one mesh (object >= 0) or of the
 * scene BVH (object == -1): BVHNode bounds/first_child/meta, nodeAreas and
 * orderedPrims (BVH.hpp:34-67, :129-135). Any output may be NULL. Returns the
 * node count, or a negative status. */
int64_t prr_scene_export_nodes(const prr_scene *scene, int object, float *bounds,
                               uint32_t *first_child, uint32_t *meta, float *areas,
                               int32_t *ordered);

/* ---- batch ray queries ------------------------------------------------- */
/* BVHAccel::Intersect on one mesh's BVH (BVH.cpp:311-415, Triangle.hpp:46-64):
 * out_id = input-order index of the closest triangle (-1 on a miss), out_t its
 * fp32 distance (+inf on a miss). out_t64 (optional) re-solves the winner's t
 * in fp64 from the input vertices (NaN on a miss). cfg may be NULL. */
int prr_mesh_intersect(const prr_scene *scene, int object, const float *o, const float *d,
                       int64_t n, int32_t *out_id, float *out_t, double *out_t64,
                       const prr_trace_config *cfg, void *stream);
/* The same with host buffers (pinned for the copies to overlap the traversal):
 * copies in, traces, copies out in chunks over the library's own streams,
 * ordered after `stream`; synchronises. cfg as for prr_mesh_intersect. */
int prr_mesh_intersect_host(prr_scene *scene, int object, const float *o, const float *d,
                            int64_t n, int32_t *out_id, float *out_t,
                            const prr_trace_config *cfg, void *stream);
/* BVHAccel::IntersectP on one mesh (BVH.cpp:421-473, Triangle.hpp:75-92):
 * out_hit[i] = 1 if an occluder lies within tmax[i]. */
int prr_mesh_occluded(const prr_scene *scene, int object, const float *o, const float *d,
                      const float *tmax, int64_t n, uint8_t *out_hit, void *stream);
/* Scene::intersect (Scene.cpp:29-31, BVH.cpp:359-369 over MeshTriangle and
 * Sphere leaves): out_obj = object index (-1 miss), out_prim = triangle index
 * within the mesh (0 for a sphere), out_t = tnear; out_geo (optional, n x 6) =
 * hit coords and geometric normal as Intersection carries them. */
int prr_scene_intersect(const prr_scene *scene, const float *o, const float *d, int64_t n,
                        int32_t *out_obj, int32_t *out_prim, float *out_t, float *out_geo,
                        void *stream);
/* Scene::intersectP (Scene.cpp:33-35, BVH.cpp:421-473 over MeshTriangle /
 * Sphere intersectT). */
int prr_scene_occluded(const prr_scene *scene, const float *o, const float *d,
                       const float *tmax, int64_t n, uint8_t *out_hit, void *stream);

/* ---- rendering --------------------------------------------------------- */
/* Renderer::Render's sample loop (Renderer.cpp:63-99) around
 * Integrator::castRay (Integrator.cpp:104-263) over the window:
 * out_rgb = window pixels x 3 floats, the linear mean radiance per pixel
 * (the framebuffer before exposure and tone mapping), row-major.
 * out_spp (optional) = samples taken per pixel; out_rays (optional, 2 x
 * uint64) = closest-hit and shadow rays traced. Device pointers. */
int prr_render(prr_scene *scene, const prr_render_settings *settings, float *out_rgb,
               int32_t *out_spp, uint64_t *out_rays, void *stream);

/* Display transform of Renderer.cpp:149-171: linear radiance times exposure,
 * non-finite and negative channels zeroed, tonemap::apply(mapper)
 * (ToneMapping.hpp:267-279), and the 8-bit quantisation
 * (unsigned char)(clamp(c,0,1)*255 + 0.5). rgb = n x 3 floats; out_rgb
 * (optional) = the mapped floats, out_u8 (optional) = n x 3 bytes. */
int prr_tonemap(int mapper, float exposure, const float *rgb, int64_t n, float *out_rgb,
                uint8_t *out_u8, void *stream);

/* The image files of Renderer::Render (Renderer.cpp:163-185): width x height
 * 8-bit RGB written to `path` as PNG (".png") or binary PPM (".ppm"). Host
 * memory. */
int prr_write_image(const char *path, const uint8_t *rgb, int width, int height);
/* The adaptive-sampling visualisation (Renderer.cpp:193-211): per pixel
 * v = (uint8)(255 * spp / max_spp) as an RGB grey. Host memory. */
int prr_sample_count_image(const int32_t *spp, int64_t n, int max_spp, uint8_t *out_rgb);

/* ---- caustic photons (PhotonMap, Photon.hpp:32-45) ---------------------- */
int prr_photon_map_create(prr_photon_map **out);
int prr_photon_map_destroy(prr_photon_map *map);
/* PhotonMap::emit + trace (Photon.cpp:96-188): num_photons photons leave the
 * scene's area emitters (photon i draws from stream (seed, i, 0xFFFFFFFF)) and
 * every diffuse hit after a specular bounce is stored. The stored records stay
 * on the device in canonical order: by emitting photon, then by trace order. */
int prr_photon_emit(prr_photon_map *map, const prr_scene *scene, int64_t num_photons,
                    uint64_t seed, int max_depth, void *stream);
/* Replaces the photon array with n records of 9 floats (position, direction,
 * power), host or device memory. */
int prr_photon_set(prr_photon_map *map, const float *records, int64_t n, void *stream);
/* PhotonMap::build -> PhotonGrid::build(caustic_map, photon_radius)
 * (Photon.cpp:24-53, :189). */
int prr_photon_build(prr_photon_map *map, float radius, void *stream);
int prr_photon_info(const prr_photon_map *map, int64_t *count, int32_t *grid_res);
/* Kernels launched so far by the calls on this photon map (emit, build,
 * gather, caustic render): a running count for launch accounting, no
 * counterpart in the reference (whose photon map runs on the host). */
int prr_photon_launches(const prr_photon_map *map, int64_t *out);
/* Copies the records (n x 9) and their emitting photon indices (n). */
int prr_photon_export(const prr_photon_map *map, float *records, int32_t *owner, void *stream);
/* PhotonMap::estimateIrradiance (Photon.cpp:82-94) at n points (n x 3):
 * sum of the powers within the radius over pi r^2. k_nearest > 0 (<= 64) caps
 * it: with more than k photons in the radius, the powers of the k nearest
 * (the k smallest (distance, photon index) pairs: of photons at equal distance
 * the lower index is kept), added in the order the grid query walks them, over
 * the disc through the k-th; identical to the fixed radius otherwise. */
int prr_photon_gather(const prr_photon_map *map, const float *points, int64_t n, int k_nearest,
                      float *out_rgb, void *stream);
/* Caustic image: for every (pixel, sample) the camera ray follows the specular
 * chain (Integrator.cpp:143-169) to its first diffuse hit x, which returns
 * beta * baseColor/pi * E(x) from the photon map. out_rgb = window x 3, each
 * pixel the mean of its samples summed in sample order. Per call, 16 bytes per
 * (pixel, sample) of at most 2^28 at once (larger renders run in chunks of
 * whole samples per pixel), 4 more with k_nearest > 0 (a queue of the
 * gathers with more than k photons inside, selected by a second kernel), come
 * from a stream-ordered memory pool of the library
 * (one per device; it keeps up to 4 GiB of freed blocks for later calls) on
 * `stream` and go back to it when the call's work is done. */
int prr_render_caustics(const prr_scene *scene, const prr_photon_map *map,
                        const prr_render_settings *settings, int k_nearest, float *out_rgb,
                        void *stream);
/* No counterpart in the reference: prr_render_caustics with counting kernels
 * (the same image), for measurement. Waits for the stream; out[0..4] = camera
 * hits traced, irradiance gathers, photons tested by the gathers' cell walks,
 * photons found inside the radius, gathers with more than k photons inside
 * (the ones the k-nearest selection runs for). */
int prr_render_caustics_counts(const prr_scene *scene, const prr_photon_map *pmap,
                               const prr_render_settings *settings, int k_nearest,
                               float *out_rgb, uint64_t out[5], void *stream);

/* ---- participating media (Volume.hpp, Volume.cpp) ----------------------
 * The reference defines a homogeneous medium and the Henyey-Greenstein phase
 * function, but its integrator never reads them (Scene::medium is not used by
 * Integrator::castRay); they are provided as batch calls over device arrays.
 * A medium is active when sigma_t > 1e-6 (Medium::active). */
typedef struct prr_medium {
    float sigma_a, sigma_s, sigma_t, g;
    int bounded;                  /* 0: the medium fills all space */
    float bounds_min[3], bounds_max[3];
} prr_medium;
#define PRR_MEDIUM_DUST 0 /* Medium::dust() */
#define PRR_MEDIUM_FOG 1  /* Medium::fog() */
int prr_medium_preset(int which, prr_medium *out);
/* Medium::intersect (Volume.hpp:17-45) of n rays (o, d: n x 3): out_hit 0/1,
 * entry and exit distances where hit (0 elsewhere). */
int prr_medium_intersect(const prr_medium *medium, const float *o, const float *d, int64_t n,
                         float *out_t_enter, float *out_t_exit, uint8_t *out_hit, void *stream);
/* phaseHG(cos_theta[k], g) (Volume.cpp:3-6). */
int prr_phase_hg(const float *cos_theta, int64_t n, float g, float *out, void *stream);
/* samplePhaseHG(wo[k], g) (Volume.cpp:8-28); item k draws from stream
 * (seed, k, 0). out_dirs: n x 3. */
int prr_phase_hg_sample(const float *wo, int64_t n, float g, uint64_t seed, float *out_dirs,
                        void *stream);

/* ---- render server: continuous batching ---------------------------------
 * No counterpart in the reference (its Renderer renders one scene per
 * process). Requests are admitted in arrival order while a slot is free and
 * the device budget (resident scenes + admitted requests) holds; every step
 * renders the next sample chunk of every running request together, so new
 * requests join running ones at the next step. */
typedef struct prr_server prr_server;
typedef struct prr_server_config {
    int64_t device_budget_bytes; /* resident scenes + admitted requests (0: 120 GiB);
                                    the step state comes on top: about 320 bytes per
                                    path of paths_per_launch, plus up to 2 GiB of
                                    pooled request blocks */
    int max_active;              /* requests rendered at once (0: 64) */
    int64_t samples_per_step;    /* megakernel steps: samples per request per step
                                    (0: 1,048,576) */
    int fail_every_nth_admission;/* fault injection on the host for tests (0: off):
                                    every n-th admission fails its allocation */
    int integrator;              /* PRR_SERVER_WAVEFRONT (0) or PRR_SERVER_MEGAKERNEL */
    int64_t paths_per_launch;    /* wavefront steps: paths per step (0: 16,777,216),
                                    a quarter shared equally among the running
                                    requests, the rest to those with the least
                                    work left */
} prr_server_config;
/* Wavefront steps: the paths of every running request share one set of
 * ordered ray queues (one traversal launch per bounce for all of them).
 * Megakernel steps: one launch over (request, 16x8 tile) items. */
#define PRR_SERVER_WAVEFRONT 0
#define PRR_SERVER_MEGAKERNEL 1
typedef struct prr_request {
    int scene;                    /* id from prr_server_add_scene */
    prr_render_settings settings; /* fixed spp (min_spp == max_spp), window, seed; width and
                                     height may differ from the scene's: the scene's camera
                                     is re-initialised for them (Camera::init) */
    float *out_rgb;               /* window x 3 floats, host or device memory */
} prr_request;
#define PRR_REQUEST_QUEUED 0
#define PRR_REQUEST_RUNNING 1
#define PRR_REQUEST_DONE 2
#define PRR_REQUEST_FAILED 3
#define PRR_REQUEST_CANCELLED 4
typedef struct prr_request_info {
    int status;                   /* PRR_REQUEST_* */
    int error;                    /* PRR_ERR_* when FAILED */
    double submit_s, admit_s, done_s; /* server steady clock, seconds */
    int64_t samples;              /* samples rendered so far */
    uint64_t rays;                /* rays traced so far */
} prr_request_info;
typedef struct prr_server_stats {
    int64_t submitted, completed, failed, active, queued;
    int64_t samples;
    uint64_t rays;
    int64_t steps;
    double busy_s;                /* time inside GPU steps */
    double admit_s;               /* worker time admitting requests (allocations) */
    double complete_s;            /* worker time resolving and returning finished images */
    int64_t bytes_in_use;
    double now_s;
    int64_t launches;             /* kernels launched by the worker so far */
} prr_server_stats;
int prr_server_create(const prr_server_config *config, prr_server **out);
/* Cancels queued requests, finishes running ones, joins the worker. */
int prr_server_destroy(prr_server *server);
/* Registers a built scene (kept resident; the caller keeps it alive until the
 * server is destroyed). All scenes are added before the first submit. */
int prr_server_add_scene(prr_server *server, prr_scene *scene, int *out_id);
int prr_server_submit(prr_server *server, const prr_request *request, uint64_t *out_id);
int prr_server_cancel(prr_server *server, uint64_t id);
int prr_server_poll(prr_server *server, uint64_t id, prr_request_info *info);
/* Blocks until the request is done, failed or cancelled (timeout_s < 0: no
 * limit); PRR_ERR_TIMEOUT otherwise. */
int prr_server_wait(prr_server *server, uint64_t id, double timeout_s, prr_request_info *info);
int prr_server_stats_get(prr_server *server, prr_server_stats *out);

/* Allocation-free rendering. No counterpart in the reference: this entry
 * point exists for callers that cannot call cudaMalloc while they render (a
 * host whose device memory is owned by another allocator, or a frame loop that
 * must not enter the CUDA allocator). It renders like prr_render in
 * PRR_RENDER_PLAIN mode with fixed spp (min_spp == max_spp), and calls no
 * cudaMalloc, cudaFree or allocating library routine: its scratch (the
 * per-slice partial sums) is a fixed device array inside the library of
 * 2,097,152 partial sums (24 MiB), held on every GPU that loads the library
 * until the process exits. Windows of more than 2,097,152 pixels are rejected
 * with PRR_ERR_INVALID_ARGUMENT, and so is an explicit settings->slices whose
 * pixels x slices exceed that count (the automatic choice, slices <= 0, is
 * reduced to fit instead). With the same settings, including the same
 * explicit slices, its image equals prr_render's bit for bit. The first call
 * on a device looks up that array's device address, so make it before any
 * stream capture. All calls
 * share the array and keep its last contents: calls that overlap on the GPU
 * race, so order them (one stream, or events). out_rays is optional. */
int prr_render_noalloc(prr_scene *scene, const prr_render_settings *settings, float *out_rgb,
                       uint64_t *out_rays, void *stream);

/* Work of one render, counted by prr_render_counts: the rays traced, the
 * traversal steps they took -- interior nodes of the scene and mesh BVHs,
 * triangle tests, object leaves (mesh entries and sphere tests) -- and the
 * closest hits by class (no hit, mirror/glass, other). */
typedef struct prr_render_count {
    uint64_t closest_rays, closest_nodes, closest_tris, closest_objects;
    uint64_t shadow_rays, shadow_nodes, shadow_tris, shadow_objects;
    uint64_t misses, delta_hits, surface_hits;
} prr_render_count;

/* No counterpart in the reference (its statistics are timings only): renders
 * like prr_render in wavefront mode (the same image) with counting variants of
 * the traversal stages, waits for the stream and fills *out. For measurement
 * (bytes per ray and per path-bounce), not for timed renders: it runs without
 * CUDA graphs and the counters cost a little. */
int prr_render_counts(prr_scene *scene, const prr_render_settings *settings, float *out_rgb,
                      prr_render_count *out, void *stream);

/* Sets the wavefront launch shape used by prr_render in wavefront mode. */
int prr_scene_set_wavefront(prr_scene *scene, const prr_wavefront_config *config);
/* The autotuner: times the wavefront renderer on `settings` (the window and
 * depth of the intended render, a few samples per pixel) over a grid of
 * paths-per-pass and block sizes with ordered queues, then, at the best of
 * those, append-order queues and shallower shared-memory stacks; keeps the
 * fastest on the scene for later renders and writes it to out_best
 * (optional). Synchronises `stream`. */
int prr_autotune(prr_scene *scene, const prr_render_settings *settings,
                 prr_wavefront_config *out_best, void *stream);

/* Integrator::castRay for a batch of (pixel, sample) pairs: the radiance of
 * each path, drawing from stream (seed, px + py*W, sample) exactly as a render
 * of that sample would. out_rgb = n x 3. */
int prr_cast_samples(const prr_scene *scene, const int32_t *px, const int32_t *py,
                     const int32_t *sample, int64_t n, uint64_t seed, int max_depth,
                     float indirect_clamp, float *out_rgb, void *stream);
/* Integrator::castRay (Integrator.cpp:104-263) for arbitrary rays (n x 3
 * origins and directions): path k draws from stream (seed, k, 0). */
int prr_cast_rays(const prr_scene *scene, const float *o, const float *d, int64_t n,
                  uint64_t seed, int max_depth, float indirect_clamp, float *out_rgb,
                  void *stream);
/* Camera::generateRay (Camera.hpp:75-95) for given pixel offsets (pinhole). */
int prr_camera_rays(const prr_scene *scene, const int32_t *px, const int32_t *py,
                    const float *xo, const float *yo, int64_t n, float *out_o, float *out_d,
                    void *stream);
/* Scene::sampleLight (Scene.cpp:37-58), sample k drawing from stream
 * (seed, k, 0): points, normals and the area pdf 1/totalEmitArea. */
int prr_scene_sample_light(const prr_scene *scene, uint64_t seed, int64_t n, float *out_pos,
                           float *out_normal, float *out_pdf, void *stream);
/* EnvMap::sample and EnvMap::importanceSamplePdf (EnvMap.hpp:97-133). */
int prr_env_eval(const prr_scene *scene, const float *dirs, int64_t n, float *out_rgb,
                 float *out_pdf, void *stream);
/* EnvMap::importanceSample (EnvMap.hpp:145-169), sample k drawing from
 * stream (seed, k, 0). */
int prr_env_importance_sample(const prr_scene *scene, uint64_t seed, int64_t n, float *out_dirs,
                              float *out_pdf, void *stream);
/* Host copies of the device-built CDF tables (EnvMap::cdf, marginalCdf,
 * totalLuminance). Any output may be NULL. */
int prr_env_export(const prr_scene *scene, float *cdf, float *marginal, float *total);

#ifdef __cplusplus
}
#endif
#endif /* PRR_H */
