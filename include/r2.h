/*
 * r2.h — C ABI of the B200-native Renderer2 hot paths (SGGX mesh-to-volume LOD
 * filter and wavefront path tracer).
 *
 * Every entry point returns an r2_status; no C++ exception crosses this
 * boundary.  Pointers are plain host pointers unless a parameter name starts
 * with `d_` (device memory on the current CUDA device).  Matrices are glm
 * column-major mat4x3 (12 floats: four columns of xyz).
 *
 * Reference interfaces replaced (paths inside FrederikBoehm/Renderer2):
 *   CConfigLoader::loadConfig        raytracer/include/backend/config_loader.hpp:36-40
 *   filter::CFilter / runFiltering   raytracer/filter.hpp:13-44, raytracer/filter.cu:20-123
 *   rt::Raytracer::renderFrame       raytracer/raytracer.hpp:29-72, raytracer/raytracer.cu:161-210
 *   CPipeline / main                 raytracer/pipeline.hpp:5-17, raytracer/main.cu:4-18
 */
#ifndef R2_H
#define R2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum r2_status {
  R2_OK = 0,
  R2_ERR_INVALID_ARGUMENT = 1,
  R2_ERR_INVALID_CONFIG = 2,
  R2_ERR_IO = 3,
  R2_ERR_OUT_OF_MEMORY = 4,
  R2_ERR_ADMISSION_REJECTED = 5,
  R2_ERR_DEVICE_TIMEOUT = 6,
  R2_ERR_DEVICE = 7,
  R2_ERR_UNSUPPORTED = 8,
  R2_ERR_NO_DEVICE = 9,
  R2_ERR_PENDING = 10  /* a served job did not finish within the wait */
} r2_status;

/* Human-readable name of a status code (static string). */
const char* r2_status_string(r2_status s);
/* Message of the last failing call on this thread ("" if none). */
const char* r2_last_error(void);
/* ABI version: major * 10000 + minor * 100 + patch. */
int r2_version(void);

/* Hierarchy of the BVHs built from now on (scenes, filter scenes, rebuilds),
 * process-wide.  Both start from the Morton-sorted primitives and end with the
 * same SAH leaf collapse.  R2_BVH_PLOC: parallel locally-ordered clustering
 * (Meister & Bittner 2018), mutual nearest neighbours by surface area within
 * 16 sorted positions.  R2_BVH_KARRAS: the radix tree of the Morton codes
 * (Karras 2012).  R2_BVH_AUTO (default): PLOC for render scenes, the Karras
 * tree for filter scenes (the faster of the two for each).  Replaces the OptiX
 * builder (optixAccelBuild, raytracer/src/mesh/mesh.cu:140-166 and
 * raytracer/src/scene/scene.cu:188-256), which has no such choice. */
enum { R2_BVH_AUTO = -1, R2_BVH_PLOC = 0, R2_BVH_KARRAS = 1 };
r2_status r2_set_bvh_method(int method);
int r2_get_bvh_method(void);

/* Voxel payload, 32 bytes, byte-identical to the reference's
 * filter::SFilteredDataCompact (raytracer/include/filtering/filtered_data.hpp:33-61),
 * which is stored in the NanoVDB Vec4d grid (openvdb_backend.cpp:27). */
typedef struct r2_voxel {
  float density;
  uint16_t sigma_x, sigma_y, sigma_z; /* [0,1] -> [0,65535] */
  uint16_t r_xy, r_xz, r_yz;          /* [-1,1] -> [0,65535] */
  uint8_t diffuse[3];
  uint8_t specular[3];
  uint16_t normal[3];                 /* [-1,1] -> [0,65535] */
  uint16_t ior;                       /* IEEE half bits */
  uint16_t pad;
} r2_voxel;

/* Surface material of a mesh: the reference's CMaterial built from MTL keys
 * (raytracer/src/material/material.cu:80-148): Kd, Ks, alpha = sqrt(2/(Ns+2)),
 * ior = Ni (1.5 when Ni == 1), Oren-Nayar roughness 0 for OBJ materials. */
typedef struct r2_material {
  float diffuse[3];
  float specular[3];
  float alpha_x, alpha_y;     /* GGX roughness */
  float eta_i, eta_t;         /* Fresnel indices (eta_t is the ior) */
  float diffuse_roughness;    /* Oren-Nayar sigma */
  float pad;
} r2_material;

/* Texture maps of a mesh's material (file paths, nullable or empty: none), as
 * the reference's CMaterial(aiMaterial*) reads them (material.cu:110-143):
 * albedo (map_Kd), specular (map_Ks; unused when the albedo map exists and a
 * specular channel is at most 0.02: the albedo's luma is the glossy colour
 * then), normal (map_Bump / bump: tangent-space normal map), alpha (map_d;
 * without it an albedo map with an alpha channel is the opacity).  Opacity 0
 * makes a triangle invisible to every ray (__anyhit__mesh,
 * shaders.optix.cu:132-152).  PNG files (any colour type). */
typedef struct r2_material_maps {
  const char* albedo;
  const char* specular;
  const char* normal;
  const char* alpha;
} r2_material_maps;

/* Filter parameters: the "Filtering" block of config.json
 * (raytracer/src/backend/config_loader.cu:75-100) plus build options. */
typedef struct r2_filter_params {
  float min_voxel_size;        /* MinVoxelSize */
  uint32_t lods;               /* LODs (voxel size doubles per LOD) */
  uint32_t samples_per_voxel;  /* SamplesPerVoxel (<= 1024) */
  float sigma_t;               /* SigmaT */
  uint32_t estimation_iterations; /* EstimationIterations */
  float alpha;                 /* Alpha */
  uint32_t clip_rays;          /* ClipRays */
  uint32_t seed;               /* Philox key word 1 */
  /* Build options without a counterpart in the reference (0: the reference's
   * plain mean of buildS).  sggx_projection 1: the mean SGGX matrix of every
   * filtered voxel is eigendecomposed in FP64 (Jacobi rotations) and replaced
   * by V diag(max(w, sggx_floor * w_max)) V^T, so that near-planar voxels
   * (one eigenvalue near 1, two near 0) keep det(S) > 0 and a finite
   * D(w) = 1/(pi sqrt|det S| (w^T S^-1 w)^2) (sggx_phase_function.hpp:107-117). */
  uint32_t sggx_projection;
  float sggx_floor;            /* relative eigenvalue floor of the projection (>= 0, < 1) */
} r2_filter_params;

/* Grid of one LOD: COpenvdbBackend::setupGrid (openvdb_backend.cpp:71-106). */
typedef struct r2_filter_grid {
  int32_t num_voxels[3];
  float index_to_model[12];
  float model_to_index[12];
  float model_to_world[12];
  float world_to_model[12];
  float world_bb_min[3];
  float world_bb_max[3];
  float voxel_size;            /* LOD voxel size (file-name suffix) */
} r2_filter_grid;

/* ------------------------------------------------------------------------ */
/* Mesh filter on host arrays (one FILTER-masked mesh, one material).
 *
 * Replaces the body of CFilter::runFiltering for one LOD
 * (raytracer/filter.cu:84-99: setupGrid, optixLaunch(nx,ny,nz), D2H copy).
 * positions: 3*nverts floats (model space); indices: 3*ntris;
 * normals: 3*nverts (model space vertex normals);
 * model_to_world: the object's T*R*S transform (12 floats);
 * voxel_size: this LOD's voxel size; out: nx*ny*nz payloads (host), indexed
 * x + y*nx + z*nx*ny.  grid_out (nullable) receives the grid.
 * wide_out (nullable): 20 floats per voxel (density, Sxx Syy Szz Sxy Sxz Syz,
 * diffuse rgb, specular rgb, normal xyz, ior, hits, mean ray length) before
 * quantisation — the parity surface against the FP64 oracle. */
r2_status r2_filter_mesh(const float* positions, uint32_t nverts, const uint32_t* indices,
                         uint32_t ntris, const float* normals, const r2_material* material,
                         const float* model_to_world, const r2_filter_params* params,
                         float voxel_size, r2_filter_grid* grid_out, r2_voxel* out,
                         float* wide_out, size_t out_capacity);

/* Grid setup only (host): world BB union, ceil(extent/vs - 0.001), transforms. */
r2_status r2_filter_setup_grid(const float* model_bb_min, const float* model_bb_max,
                               const float* model_to_world, float voxel_size,
                               r2_filter_grid* grid_out);

/* ------------------------------------------------------------------------ */
/* Device-resident filter scene (inputs stay in HBM between launches). */
typedef struct r2_filter_scene r2_filter_scene;

r2_status r2_filter_scene_create(const float* positions, uint32_t nverts,
                                 const uint32_t* indices, uint32_t ntris, const float* normals,
                                 const r2_material* material, const float* model_to_world,
                                 r2_filter_scene** out);
/* The same with texture coordinates (2 per vertex) and the material's texture
 * maps (see r2_material_maps): each hit contributes diffuse(tc), glossy(tc)
 * and the normal-mapped normal, and opacity cut-outs hide triangles from the
 * filter rays (CMeshFilter::run, mesh_filter.hpp:300-371, over the closest-hit
 * and any-hit programs, shaders.optix.cu:28-152). */
r2_status r2_filter_scene_create_textured(const float* positions, uint32_t nverts, const uint32_t* indices,
                                          uint32_t ntris, const float* normals, const float* uvs,
                                          const r2_material* material, const r2_material_maps* maps,
                                          const float* model_to_world, r2_filter_scene** out);
r2_status r2_filter_scene_destroy(r2_filter_scene* scene);
/* Grid for a voxel size over this scene's bounds. */
r2_status r2_filter_scene_grid(const r2_filter_scene* scene, float voxel_size,
                               r2_filter_grid* grid_out);
/* Filter one LOD into device memory.  d_out: nx*ny*nz r2_voxel; d_wide
 * (nullable): 20 floats per voxel; d_fp16 (nullable): 8 halves per voxel
 * (density, Sxx, Syy, Szz, Sxy, Sxz, Syz, 0).  stream: cudaStream_t or NULL.
 * stats_out (nullable, host): [0]=voxels, [1]=voxels with candidate geometry,
 * [2]=kernel milliseconds of the per-voxel sampling kernel. */
r2_status r2_filter_scene_run(r2_filter_scene* scene, const r2_filter_grid* grid,
                              const r2_filter_params* params, r2_voxel* d_out, float* d_wide,
                              uint16_t* d_fp16, void* stream, double* stats_out);
/* The same with the FP64 eigendecomposition of each voxel's SGGX matrix:
 * d_eig (device, 12 floats per voxel) receives w0 >= w1 >= w2, then the unit
 * eigenvectors v0, v1, v2 (3 floats each, largest-magnitude entry
 * non-negative) of the mean S before any projection; zeros for voxels without
 * hits.  The rest of the output is that of r2_filter_scene_run, bit for bit.
 * The reference stores S and never decomposes it. */
r2_status r2_filter_scene_run_eig(r2_filter_scene* scene, const r2_filter_grid* grid,
                                  const r2_filter_params* params, r2_voxel* d_out, float* d_wide,
                                  uint16_t* d_fp16, float* d_eig, void* stream, double* stats_out);
/* The same LOD through the counting build of the sampling kernel (same
 * payloads, slower): counts_out[0] rays traced, [1] inner BVH nodes visited,
 * [2] triangles tested -- the operation counts behind the filter's
 * arithmetic roofline.  Waits for the result. */
r2_status r2_filter_scene_count(r2_filter_scene* scene, const r2_filter_grid* grid,
                                const r2_filter_params* params, r2_voxel* d_out, uint64_t* counts_out);

/* Same as r2_filter_scene_run, for callers that must not allocate device
 * memory during the call: frame loops that run under a fixed memory budget
 * with no allocation after start-up, applications that own every device
 * allocation through their own pool, and latency-bound callers that cannot
 * afford the device-wide synchronisation cudaMalloc/cudaFree may imply.
 * It allocates nothing: the voxel work list and queue counters live in a
 * fixed scratch array inside the library (4 MiB, held by every GPU that loads
 * the library until the process exits), so grids above 2^20 voxels are
 * rejected with R2_ERR_UNSUPPORTED.  The scene is created beforehand with
 * r2_filter_scene_create.  The first call on a device resolves the scratch
 * array's device address (set-up done once per device) and should come
 * before any stream capture.  All calls share the one scratch array and it
 * keeps the last call's contents: calls that overlap on the GPU race and must
 * be serialised by the caller.  stream NULL means the device's legacy default
 * stream (not the scene's private stream), so calls given NULL run one after
 * another, whichever scene each filters.  The current device, and the device
 * of a given stream, must be the scene's device (R2_ERR_INVALID_ARGUMENT
 * otherwise).
 * This entry point has no counterpart in the reference. */
r2_status r2_filter_scene_run_static(r2_filter_scene* scene, const r2_filter_grid* grid,
                                     const r2_filter_params* params, r2_voxel* d_out, float* d_wide,
                                     uint16_t* d_fp16, void* stream);

/* All LODs with the reference's file outputs (CFilter::runFiltering,
 * raytracer/filter.cu:74-123): voxel size min_voxel_size * 2^lod; per LOD
 * <out_root>/<model_name>/filtered_mesh_<std::to_string(vs)>.nvdb (NanoVDB
 * Vec4d grid, active = density > 0 or a grid corner, openvdb_backend.cpp:108-157)
 * and .brickgrid (density bricks + majorant mips, host_grid_brick.cpp:61-152),
 * and <out_root>/volume_description.json (volume_description_manager.cpp:50-144).
 * The object transform is T(pos3) * getRotation(orientation3) * S(scaling3)
 * (src/scene/sceneobject.cu:375-377).  stats_out (nullable, 4 doubles): LODs,
 * voxels, active voxels, sampling-kernel milliseconds. */
r2_status r2_filter_run_mesh(const float* positions, uint32_t nverts, const uint32_t* indices, uint32_t ntris,
                             const float* normals, const r2_material* material, const float* pos3,
                             const float* orientation3, const float* scaling3, const r2_filter_params* params,
                             const char* out_root, const char* model_name, double* stats_out);

/* NanoVDB file written by the filter: counts4 = leaves, lower nodes, upper
 * nodes, active voxels; index_bbox6 = active index box (inclusive);
 * world_bbox6; index_to_model12 = the grid map as a glm mat4x3. */
r2_status r2_nvdb_info(const char* path, uint64_t* counts4, int32_t* index_bbox6, double* world_bbox6,
                       float* index_to_model12);
/* Payloads and active flags at n index coordinates (3 int32 each). */
r2_status r2_nvdb_lookup(const char* path, const int32_t* coords, uint32_t n, r2_voxel* out, uint8_t* active);
/* Brick grid file: dims7 = bricks xyz, atlas voxels xyz, non-constant bricks;
 * minmaj2 = density minorant/majorant; indirection/range (nullable) receive
 * the per-brick words (capacity in elements). */
r2_status r2_brickgrid_info(const char* path, uint32_t* dims7, float* minmaj2, uint32_t* indirection,
                            uint32_t* range, size_t capacity);

/* BVH of a filter scene, downloaded for bit-exact comparison with the oracle:
 * nodes: (ntris-1 or 1) * 16 words; tri_order: ntris original indices. */
r2_status r2_filter_scene_bvh(const r2_filter_scene* scene, int32_t* nodes, size_t node_words,
                              uint32_t* tri_order, size_t ntris, uint32_t* nnodes_out,
                              uint32_t* height_out);

/* ------------------------------------------------------------------------ */
/* Path tracer.
 *
 * Replaces rt::Raytracer (raytracer/raytracer.hpp:29-72): construction
 * (raytracer.cu:129-152: scene upload, acceleration structure, samplers) and
 * renderFrame (raytracer.cu:161-210: clear, one launch per sample of
 * CPathIntegrator::Li, include/integrators/path_integrator_impl.hpp:120-247).
 * The acceleration structure is this library's LBVH (no OptiX).  The frame
 * is the linear, pre-tonemap radiance buffer of SFrame::data
 * (common/frame.hpp:6-12): 3 floats per pixel, row 0 at the bottom. */
typedef struct r2_scene r2_scene;

/* CCamera(sensorWidth, sensorHeight, fov, pos, lookAt, up)
 * (raytracer/include/camera/camera.hpp:27): fov is the horizontal FOV in degrees. */
typedef struct r2_camera {
  uint32_t width, height;
  float fov_deg;
  float pos[3];
  float look_at[3];
  float up[3];
} r2_camera;

typedef struct r2_render_params {
  uint32_t spp;        /* "Samples" of config.json */
  uint32_t max_depth;  /* bounce cap (the reference hard-codes 50) */
  uint32_t seed;       /* Philox key word 1 */
  uint32_t flags;      /* R2_RENDER_* bits */
} r2_render_params;

/* Launch tuning of a scene's renders.  No image depends on it: every setting
 * gives the same frames bit for bit.  0 selects the built-in default. */
typedef struct r2_render_tuning {
  uint32_t track_steps; /* media: tracking steps a lane of the persistent tracker takes between refills (1..1024) */
  uint32_t trav_visits; /* BVH node/leaf visits a lane takes between refill checks of the surface kernels */
  uint32_t trav_refill; /* finished lanes of a warp (1..32) that make it take new rays */
  uint32_t wave_paths;  /* paths per wave: a wave renders the largest divisor of spp samples of every
                           pixel that keeps width*height*samples within it (at least one sample) */
  uint32_t media_rounds; /* media: queued rounds of medium boundaries per bounce (1..32) before the
                            remaining boundaries of a path are walked in one pass */
  uint32_t track_blocks; /* media: blocks per SM of the persistent trackers (at most the resident
                            blocks; 0: all of them) */
  uint32_t track_limit; /* media: bound on the steps of one tracking loop (delta / ratio tracking of
                           one medium segment; 0: 2^20, the maximum).  A safety bound, not a tuning:
                           a path or shadow ray whose loop reaches it ends, and the synchronous
                           render calls return R2_ERR_DEVICE_TIMEOUT with the frame written.  The
                           reference's loops have no bound (nvdb_medium_impl.hpp:98-136, 155-186). */
  uint32_t top_nodes;   /* surface scenes: BVH nodes 0 .. top_nodes-1 copied into each traversal block's
                           shared memory and read from there (0: off; at most 256).  With the PLOC
                           builder a parent's index is below its children's, so these are the top
                           levels of the tree (of the top-level tree in two-level scenes). */
  uint32_t sort_rays;   /* surface scenes: 1 reorders each bounce's rays after the first by direction
                           octant, dominant axis and origin cell before tracing them (a counting sort
                           over 256 keys); 0: off.  The order of rays changes no bit of a frame. */
} r2_render_tuning;

/* "UseBrickGrid" of config.json: media are tracked with the brick-grid DDA
 * (CNVDBMedium::sampleDDA / trDDA, nvdb_medium_impl.hpp:139-187, 248-294)
 * instead of the global majorant (sampleInternal / trInternal, 94-137, 203-239). */
#define R2_RENDER_BRICK_GRID 1u

/* Object masks (raytracer/include/scene/sceneobject_mask.hpp:6-11). */
#define R2_MASK_FILTER 1u
#define R2_MASK_RENDER 2u
#define R2_MASK_ALL 255u

/* Analytic shapes of scenedescription.json (Type "Sphere" / "Circle"). */
#define R2_SHAPE_SPHERE 0
#define R2_SHAPE_CIRCLE 1

r2_status r2_scene_create(r2_scene** out);
r2_status r2_scene_destroy(r2_scene* scene);
/* Adds a triangle mesh (model space) with one material and its T*R*S transform. */
r2_status r2_scene_add_mesh(r2_scene* scene, const float* positions, uint32_t nverts, const uint32_t* indices,
                            uint32_t ntris, const float* normals, const r2_material* material,
                            const float* model_to_world, uint32_t mask);
/* Instanced meshes (two-level scenes).  r2_scene_add_mesh_asset keeps a mesh
 * in model space with its own BVH (uvs and maps nullable, as
 * r2_scene_add_mesh_textured) and returns its index; r2_scene_add_mesh_instance
 * places it with a T*R*S transform (mask 0: not visible to render rays).
 * Once a scene has an instance, the BVH becomes two-level: a top level over
 * the instances' world boxes (the world-space meshes of r2_scene_add_mesh
 * form one more instance) and one bottom level per asset, each shared by its
 * instances.  Replaces CAssetManager::loadMesh's per-file mesh with its GAS
 * and the scene objects' OptiX instances (raytracer/src/scene/scene.cu:188-256,
 * raytracer/src/scene/sceneobject.cu:330-349): a hit's normal is the
 * interpolated model-space normal taken to world space by the instance's
 * transform (__closesthit__ch, shaders.optix.cu:28-130).  Assets do not
 * change after commit; r2_scene_set_vertices and r2_scene_rebuild act on the
 * world-space meshes and rebuild the top level. */
r2_status r2_scene_add_mesh_asset(r2_scene* scene, const float* positions, uint32_t nverts, const uint32_t* indices,
                                  uint32_t ntris, const float* normals, const float* uvs, const r2_material* material,
                                  const r2_material_maps* maps, uint32_t* asset_out);
r2_status r2_scene_add_mesh_instance(r2_scene* scene, uint32_t asset, const float* model_to_world, uint32_t mask);
r2_status r2_scene_add_shape(r2_scene* scene, int shape_type, const float* center, float radius,
                             const float* normal, const r2_material* material, uint32_t mask);
/* Environment map: width*height RGB float texels, row 0 = top (+Y). */
r2_status r2_scene_set_envmap(r2_scene* scene, const float* rgb, uint32_t width, uint32_t height);
/* Heterogeneous SGGX medium of scenedescription.json (Type "Medium"): loads
 * <path>.nvdb and <path>.brickgrid (path without extension, ending in the
 * filter voxel size "\d+.\d+"), placed with T(pos) R(orientation) S(scaling).
 * Replaces CNVDBMedium(path, sigma_a, sigma_s) (raytracer/src/medium/nvdb_medium.cu:45-61,
 * 130-173) inside CHostSceneobject(medium, pos, orientation, scaling, mask)
 * (raytracer/src/scene/sceneobject.cu:50-65). */
r2_status r2_scene_add_medium(r2_scene* scene, const char* path, const float* sigma_a, const float* sigma_s,
                              const float* pos, const float* orientation, const float* scaling, uint32_t mask);
/* Same with the Henyey-Greenstein phase function of asymmetry g (Medium with a
 * "G" key; CNVDBMedium(path, sigma_a, sigma_s, g), nvdb_medium.cu:27-43). */
r2_status r2_scene_add_medium_hg(r2_scene* scene, const char* path, const float* sigma_a, const float* sigma_s,
                                 float g, const float* pos, const float* orientation, const float* scaling,
                                 uint32_t mask);
/* r2_scene_add_mesh with texture coordinates (uvs: 2 per vertex, v = 0 at the
 * maps' top row as stb_image loads them) and texture maps. */
r2_status r2_scene_add_mesh_textured(r2_scene* scene, const float* positions, uint32_t nverts, const uint32_t* indices,
                                     uint32_t ntris, const float* normals, const float* uvs,
                                     const r2_material* material, const r2_material_maps* maps,
                                     const float* model_to_world, uint32_t mask);
/* Uploads the scene and builds the BVH (device-resident until destroyed). */
r2_status r2_scene_commit(r2_scene* scene);
/* Rebuilds the committed scene's triangle BVH on the device from its resident
 * triangles, on `stream` (cudaStream_t; NULL: the scene's own stream), and
 * re-gathers the per-triangle shading data in the new leaf order: the
 * acceleration-structure build of CHostScene::buildOptixAccel
 * (raytracer/src/scene/scene.cu:188-256, mesh.cu:140-168) done per frame,
 * with the geometry already in device memory.  The tree equals the commit's;
 * nothing is allocated after the first build; the call returns once the
 * build has finished on the device.  Frames must not be rendering the scene
 * on another stream meanwhile. */
r2_status r2_scene_rebuild(r2_scene* scene, void* stream);
/* The surface BVH of a committed scene: inner nodes, height (levels of inner
 * nodes on the longest path) and the kernels its last build or rebuild
 * launched.  Any output may be NULL. */
r2_status r2_scene_bvh_info(r2_scene* scene, uint32_t* nodes, uint32_t* height, uint32_t* build_launches);

/* Replaces the committed scene's vertex positions (and, when normals is not
 * NULL, its vertex normals) with nverts world-space vertices from host memory
 * (pinned memory makes the copy asynchronous), in the order the meshes were
 * added: the per-frame geometry upload of a dynamic scene.  Triangles,
 * materials and the vertex count stay; call r2_scene_rebuild before the next
 * frame.  stream as in r2_scene_rebuild; the host arrays must stay valid
 * until the stream has copied them. */
r2_status r2_scene_set_vertices(r2_scene* scene, const float* positions, const float* normals, uint32_t nverts,
                                void* stream);
/* Renders one frame into device memory d_rgb (width*height*3 floats).
 * stats_out (nullable, 8 doubles): [0] paths, [1] milliseconds of the frame on
 * the stream, [2] path segments traced, [3] shadow rays traced, [4..7]
 * milliseconds of the extend / shade / shadow / accumulate kernels of one
 * (the middle) wave, which renders r2_scene_wave_samples samples of every
 * pixel.  With stats_out the call waits for the frame and returns
 * R2_ERR_DEVICE_TIMEOUT (frame still written) if a loop bound ended any path:
 * 2^20 tracking steps, 64 medium boundaries within a bounce, 256 along a
 * shadow ray (the reference's loops have no bound). */
r2_status r2_render_device(r2_scene* scene, const r2_camera* camera, const r2_render_params* params, float* d_rgb,
                           void* stream, double* stats_out);
/* Same through host memory: commits if needed, renders into a device frame
 * the scene keeps (grown on demand, reused by later calls), copies the frame
 * to rgb and waits; loop bounds are reported as in r2_render_device. */
r2_status r2_render_host(r2_scene* scene, const r2_camera* camera, const r2_render_params* params, float* rgb);

/* The scene's launch tuning (initially the defaults, or the environment's
 * R2_TRACK_STEPS / R2_TRAV_VISITS / R2_TRAV_REFILL). */
r2_status r2_scene_set_tuning(r2_scene* scene, const r2_render_tuning* tuning);
r2_status r2_scene_get_tuning(r2_scene* scene, r2_render_tuning* tuning);
/* Samples of every pixel that one wave of this frame renders under the
 * scene's tuning (stats_out[4..7] of r2_render_device time one such wave). */
r2_status r2_scene_wave_samples(r2_scene* scene, const r2_camera* camera, const r2_render_params* params,
                                uint32_t* samples_out);
/* Autotuner: times one wave of this frame for each candidate value of one
 * setting at a time (scenes without media: refill lanes, then visits; with
 * media: tracking steps), keeps a candidate that is faster by more than 2 %,
 * and stores the result as the scene's tuning (also written to tuning_out,
 * nullable).  Commits the scene if needed; waits. */
r2_status r2_scene_autotune(r2_scene* scene, const r2_camera* camera, const r2_render_params* params,
                            r2_render_tuning* tuning_out);

/* Frames of n committed scenes (a scene may appear more than once) rendered
 * together by one captured CUDA graph holding one wave of every frame, each on
 * a branch of its own so that their kernels overlap; the graph is replayed
 * once per sample.  The reference renders one scene per process
 * (CPipeline::run, pipeline.cu:18-90); a batch is how many scenes share one
 * GPU.  Every frame equals r2_render_device's with the same arguments.
 * Cameras, parameters (all with the same spp) and device frames d_rgb[i]
 * (width*height*3 floats) are fixed at creation; the scenes must outlive the
 * batch. */
typedef struct r2_render_batch r2_render_batch;
r2_status r2_render_batch_create(r2_scene* const* scenes, const r2_camera* cameras, const r2_render_params* params,
                                 float* const* d_rgb, uint32_t n, r2_render_batch** out);
r2_status r2_render_batch_destroy(r2_render_batch* batch);
/* Clears and renders every frame on stream (null: the default stream).  With
 * ms_out the call waits, stores the device milliseconds of all samples and
 * returns R2_ERR_DEVICE_TIMEOUT (frames still written) if a loop bound ended
 * any path, as r2_render_device does. */
r2_status r2_render_batch_run(r2_render_batch* batch, void* stream, double* ms_out);

/* ------------------------------------------------------------------------ */
/* Pipeline: config.json + scenedescription.json.
 *
 * Replaces CConfigLoader::loadConfig (raytracer/include/backend/config_loader.hpp:36-40,
 * raytracer/src/backend/config_loader.cu:340-368) and CPipeline(configPath) / run()
 * (raytracer/pipeline.hpp:5-17, pipeline.cu:18-90).  Loading parses both JSON
 * files (comments allowed), reads the Radiance .hdr environment map and the
 * OBJ/MTL meshes; media are read at the first render.  Relative paths resolve
 * against the working directory, as in the reference. */
typedef struct r2_config r2_config;

typedef struct r2_config_info {
  uint32_t frame_width, frame_height, channels, samples;  /* General */
  float gamma;
  uint32_t use_brick_grid;
  uint32_t filter_active;                                  /* Filtering.Active */
  r2_filter_params filter;                                 /* Filtering (seed 0) */
  r2_camera camera;                                        /* Camera */
  uint32_t env_width, env_height;                          /* Scene.Envmap */
  uint32_t n_shapes, n_meshes, n_media;                    /* n_meshes counts OBJ submeshes */
  uint32_t n_triangles;
} r2_config_info;

typedef struct r2_render_opts {
  uint32_t spp;        /* 0: General.Samples */
  uint32_t max_depth;  /* 0: 50, the reference's bounce cap */
  uint32_t seed;
  uint32_t flags;      /* reserved, 0 */
} r2_render_opts;

r2_status r2_config_load(const char* config_json_path, r2_config** out);
r2_status r2_config_free(r2_config* cfg);
r2_status r2_config_info_get(const r2_config* cfg, r2_config_info* out);
/* CFilter(config).runFiltering() (raytracer/filter.hpp:183-214, filter.cu:20-123):
 * the FILTER-masked mesh (one OBJ file, all its submeshes) filtered for every
 * LOD into <out_root>/<mesh name>/filtered_mesh_<vs>.{nvdb,brickgrid} and
 * <out_root>/volume_description.json; out_root NULL means "./filtering".
 * Without FILTER objects nothing is written (R2_OK).  stats_out (nullable, 4
 * doubles): LODs, voxels, active voxels, kernel milliseconds. */
r2_status r2_filter_run(r2_config* cfg, const char* out_root, double* stats_out);
/* Raytracer(config).renderFrame() (raytracer/raytracer.hpp:29-72,
 * raytracer.cu:161-210): the scene stays resident on the device across calls.
 * out_linear_rgb (nullable): W*H*3 pre-tonemap radiance, row 0 at the bottom;
 * out_bytes (nullable): W*H*3 bytes after the log-average tonemap and gamma
 * (SFrame::dataBytes). */
r2_status r2_render(r2_config* cfg, const r2_render_opts* opts, float* out_linear_rgb, uint8_t* out_bytes);
/* Output stage on host buffers (raytracer.cu:33-127): L = exp(sum log(r+g+b+FLT_MIN)
 * / (3WH)) - WH FLT_MIN; c / (c + L); ^(1/gamma); bytes = round(255 c). */
r2_status r2_tonemap(const float* linear_rgb, uint32_t width, uint32_t height, float gamma, float* out_rgb,
                     uint8_t* out_bytes);
/* Image files: 8-bit RGB PNG (flip_vertical as the reference's writer does for
 * bottom-up frames) and Radiance RGBE .hdr (row 0 = top). */
r2_status r2_write_png(const char* path, const uint8_t* rgb, uint32_t width, uint32_t height, int flip_vertical);
/* Baseline JPEG (4:4:4, standard tables, quality 1..100): the output.jpg of
 * CImageWriter::writeToFile (visualisation/src/image_writer.cpp:13-17, quality 100). */
r2_status r2_write_jpg(const char* path, const uint8_t* rgb, uint32_t width, uint32_t height, int flip_vertical,
                       int quality);
r2_status r2_read_hdr(const char* path, float* rgb, size_t capacity, uint32_t* width, uint32_t* height);
/* PNG texture (any colour type, 1-16 bits, non-interlaced) as 8-bit RGBA, row 0 = top,
 * as stb_image loads the reference's texture maps (texture.cu:64-97).  rgba may be
 * null to query the size; channels_out: the file's channel count (1-4). */
r2_status r2_read_png(const char* path, uint8_t* rgba, size_t capacity, uint32_t* width, uint32_t* height,
                      int* channels_out);
r2_status r2_write_hdr(const char* path, const float* rgb, uint32_t width, uint32_t height);
/* OBJ/MTL import summary (CAssetManager::loadWithAssimp, asset_manager.cu:25-84). */
r2_status r2_obj_info(const char* directory, const char* filename, uint32_t* n_submeshes, uint32_t* n_vertices,
                      uint32_t* n_triangles, r2_material* first_material);

/* ------------------------------------------------------------------------ */
/* Screen-space LOD selection for many-instance scenes: the forest generator's
 * selectLOD (raytracer/src/filtering/generate_random_forest.py:179-225, with
 * project 73-80, projectLOD 82-101, outsideFrustum 103-105, gamma 132-133,
 * intersectBB 135-151, approximateNumVoxels2 153-177), one GPU thread per
 * tree, in double precision like the generator's numpy.
 *
 * Per tree: if all 8 projected corners of the model's coarsest LOD lie outside
 * the frustum the coarsest LOD is chosen; otherwise the convex hull area of
 * the projected corners gives the covered pixels, and the LODs of voxel size
 * >= min_lod are walked in the order given (the generator's sorted(lods):
 * the volume description's keys in string order); each one whose estimated
 * visible voxel count times covered_pixels exceeds the covered pixels
 * becomes the choice, the first that does not ends the walk.  The choice -1
 * means the mesh itself (the generator's "0"). */
typedef struct r2_lod_camera {
  double world_to_view[16];    /* row-major 4x4 (common_functions.py lookAt) */
  double pos[3];
  double near_plane_distance;  /* sensor_width * pixel_size / (2 tan(fov / 2)) */
  double pixel_size;           /* 1e-5 in the generator */
  double pixel_area;           /* pixel_size ** 2 as the host computes it */
  double sensor_width, sensor_height;
  double far_scale;            /* intersectBB's far-distance factor 1 + 2 gamma(3) */
} r2_lod_camera;

/* One LOD of a model: an entry of volume_description.json. */
typedef struct r2_lod_volume {
  double voxel_size;     /* the entry's key as a number */
  double bb_min[3], bb_max[3];
  double num_voxels[3];
  double corners[8][3];  /* P0..P7 */
} r2_lod_volume;

/* lods: all models' LODs, model m's at [model_first[m], model_first[m] +
 * model_count[m]) in walk order; trees: position (3 doubles), uniform
 * scaling, model index.  lod_out (ntrees): index into lods, or -1 for the
 * mesh.  Host buffers; the selection runs on the current device. */
r2_status r2_select_lods(const r2_lod_camera* camera, const r2_lod_volume* lods, const uint32_t* model_first,
                         const uint32_t* model_count, uint32_t nmodels, const double* tree_pos,
                         const double* tree_scaling, const uint32_t* tree_model, uint32_t ntrees, double min_lod,
                         double covered_pixels, int32_t* lod_out);

/* ------------------------------------------------------------------------ */
/* Serving: a request loop that overlaps jobs on the device (continuous
 * batching).  This has no counterpart in the reference, which renders one
 * frame at a time (raytracer/pipeline.cu:24-90).
 *
 * Jobs wait in a FIFO queue; the loop admits the head as soon as one of
 * `slots` slots is free and the job's device memory (wave state and frame, or
 * voxel output and work list) fits in what `hbm_budget_bytes` leaves.  Each
 * slot has its own stream and buffers; scenes stay resident and must stay
 * alive and unmodified (committed) while their jobs run.  Each result is the
 * same alone and in any mix (random streams depend on pixel, sample and seed
 * only).  A job's output is written to the caller's buffer before r2_server_wait
 * reports it. */
typedef struct r2_server r2_server;
r2_status r2_server_create(uint32_t slots, uint64_t hbm_budget_bytes, r2_server** out);
/* Finishes admitted and queued jobs, then releases the server. */
r2_status r2_server_destroy(r2_server* server);
/* A frame of a committed scene into rgb_out (W*H*3 floats, row 0 at the bottom).
 * R2_ERR_ADMISSION_REJECTED if the job alone exceeds the budget. */
/* Device bytes a render job of this scene, camera and parameters is admitted
 * with (checked against the budget; plan budgets with it). */
r2_status r2_server_render_bytes(r2_scene* scene, const r2_camera* camera, const r2_render_params* params,
                                 uint64_t* bytes_out);
r2_status r2_server_submit_render(r2_server* server, r2_scene* scene, const r2_camera* camera,
                                  const r2_render_params* params, float* rgb_out, uint64_t* job_id);
/* One LOD of a filter scene into out (nx*ny*nz payloads). */
r2_status r2_server_submit_filter(r2_server* server, r2_filter_scene* scene, const r2_filter_grid* grid,
                                  const r2_filter_params* params, uint32_t lod, r2_voxel* out, uint64_t* job_id);
/* Waits up to timeout_s seconds (< 0: forever).  Returns R2_ERR_PENDING if the
 * job is not done yet (it can be waited for again), else the job's own status;
 * times_out (nullable, 3 doubles): submit, start and end times in seconds on the
 * server's clock.  A finished job is forgotten once waited for. */
r2_status r2_server_wait(r2_server* server, uint64_t job_id, double timeout_s, double* times_out);
/* stats_out (5 doubles): jobs done, jobs queued, jobs running, device bytes
 * admitted, seconds since the server started. */
r2_status r2_server_stats(r2_server* server, double* stats_out);

#ifdef __cplusplus
}
#endif

#endif /* R2_H */
