/*
 * CPU oracle for the Renderer2 hot paths — TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm may load this library, and only as the checker or the timed CPU
 * baseline; the product path never calls it.
 *
 * It restates, in plain C, the reference algorithms of FrederikBoehm/Renderer2:
 *   - per-voxel SGGX filtering, CMeshFilter::run / estimateDensity
 *     (raytracer/include/filtering/mesh_filter.hpp:51-122, 182-226);
 *   - the 32-byte payload encode, SFilteredDataCompact(const SFilteredData&)
 *     (raytracer/include/filtering/filtered_data.hpp:91-107);
 *   - SGGX S construction, buildS (raytracer/include/medium/sggx_phase_function.hpp:95-105);
 *   - the bounding-sphere clip, Sphere::intersect (raytracer/include/shapes/sphere.hpp:33-90);
 *   - grid setup, COpenvdbBackend::setupGrid (raytracer/src/filtering/openvdb_backend.cpp:71-106);
 * driven by the same Philox4x32-10 streams as the GPU kernels, over its own
 * LBVH built with the same deterministic algorithm (bit-exact leaf assignment).
 * Geometry (ray generation, traversal, hit normals) is FP32 with the same
 * operation order as the device code; accumulation, the density fit and the
 * mean normal are FP64 (the "FP64 rebuild").
 *
 * Parity pinning: the reference has no tests or golden vectors, and its own
 * RNG (cuRAND XORWOW) and OptiX traversal cannot run here.  The math functions
 * this oracle restates are pinned against the reference's own headers compiled
 * for the host (oracle/ref_kat.cpp -> oracle/_ref/libr2ref.so) through the
 * golden vectors in tests/golden/.
 */
#ifndef R2_ORACLE_H
#define R2_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_sincos_turns(float u, float* s, float* c);

/* BVH identical to the GPU builder (method: orc_set_bvh_method).  nodes_out: (ntris > 1 ? ntris-1 : 1) * 16
 * int32 words (BvhNode layout), order_out: ntris.  Returns the tree height or
 * -1 on error. */
int orc_build_bvh(const float* world_pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris,
                  int32_t* nodes_out, uint32_t* order_out, float* tris_out /* 12*ntris or NULL */);

/* Hierarchy of the BVHs built from now on: 0 PLOC clustering, 1 the Karras
 * radix tree, -1 (default) PLOC for render scenes and Karras for filter
 * scenes; the GPU builder's methods. */
void orc_set_bvh_method(int method);
int orc_get_bvh_method(void);
/* orc_build_bvh for a filter scene (its default hierarchy under -1). */
int orc_build_bvh_filter(const float* world_pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris,
                         int32_t* nodes_out, uint32_t* order_out, float* tris_out);

/* Closest hit: returns BVH-order triangle or -1; t/b1/b2 out. */
int orc_trace(const int32_t* nodes, const float* tris, float ox, float oy, float oz, float dx, float dy,
              float dz, float tmax, float* t, float* b1, float* b2);

typedef struct orc_material {
  float diffuse[3];
  float specular[3];
  float alpha_x, alpha_y, eta_i, eta_t, diffuse_roughness, pad;
} orc_material;

typedef struct orc_filter_params {
  float min_voxel_size;
  uint32_t lods;
  uint32_t samples_per_voxel;
  float sigma_t;
  uint32_t estimation_iterations;
  float alpha;
  uint32_t clip_rays;
  uint32_t seed;
  uint32_t sggx_projection; /* 1: S replaced by its eigen-projection with eigenvalues >= sggx_floor * max */
  float sggx_floor;
} orc_filter_params;

typedef struct orc_grid {
  int32_t num_voxels[3];
  float index_to_model[12];
  float model_to_index[12];
  float model_to_world[12];
  float world_to_model[12];
  float world_bb_min[3];
  float world_bb_max[3];
  float voxel_size;
} orc_grid;

/* Grid setup from the model bounds and the object's model_to_world. */
void orc_setup_grid(const float* model_lo, const float* model_hi, const float* model_to_world, float voxel_size,
                    orc_grid* g);

/* A texture map as decoded from its file: 8-bit RGBA, row 0 = top, and the
 * file's channel count. */
typedef struct orc_texture {
  uint32_t width, height;
  int channels;
  const uint8_t* rgba;
} orc_texture;

/* Filters voxels [v0, v1) of the grid.  wide_out: 20 doubles per voxel of the
 * range (density, S xx yy zz xy xz yz, diffuse, specular, normal, ior, hits,
 * mean ray length, mean roughness); compact_out: 32 bytes per voxel of the
 * range (nullable).  threads: worker threads (0 = all cores).  The mesh is in
 * model space; positions and hit normals use obj_model_to_world (the
 * object's own transform), voxel centres the grid's model_to_world.  lod is
 * the Philox counter word of the LOD. */
int orc_filter(const float* positions, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* normals,
               const orc_material* mat, const float* obj_model_to_world, const orc_grid* g,
               const orc_filter_params* p, uint32_t lod, uint64_t v0, uint64_t v1, double* wide_out,
               uint8_t* compact_out, int threads);
/* The same for a textured material: uvs (2 per vertex) and the texture maps
 * (nullable each; map_Kd, map_Ks, map_Bump, map_d as CMaterial(aiMaterial*)
 * reads them, material.cu:110-143). */
int orc_filter_tex(const float* positions, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* normals,
                   const float* uvs, const orc_material* mat, const orc_texture* albedo, const orc_texture* specular,
                   const orc_texture* normal, const orc_texture* alpha, const float* obj_model_to_world,
                   const orc_grid* g, const orc_filter_params* p, uint32_t lod, uint64_t v0, uint64_t v1,
                   double* wide_out, uint8_t* compact_out, int threads);

/* Eigendecomposition of the symmetric 3x3 S (xx yy zz xy xz yz) in double by
 * cyclic Jacobi rotations: w descending, V row-major (V[3*row + col]) with
 * unit eigenvector columns, each with its largest-magnitude entry >= 0. */
void orc_sym3_eig(const double* S6, double* w3, double* V9);

/* CHostBrickGrid construction (brick_oracle.c) from the grid's densities
 * (nx*ny*nz floats, x fastest, inactive voxels 0): n_bricks in nb (3); with
 * ind null only nb is computed.  ind, range: nb products; mip0..2:
 * (nb >> (i+1)) products; atlas: capacity nb*8 per axis (zeroed here); ad:
 * atlas dims after the z prune; count: bricks with an atlas slot; minmaj: the
 * grid's density min and max.  Returns -1 beyond 1023 bricks per axis. */
int orc_build_bricks(const float* dens, int nx, int ny, int nz, uint32_t* nb, uint32_t* ind, uint32_t* range,
                     uint32_t* mip0, uint32_t* mip1, uint32_t* mip2, uint8_t* atlas, uint32_t* ad,
                     uint64_t* count, float* minmaj);

/* Encode a wide (double) record to the 32-byte payload (FP64 arithmetic). */
void orc_encode(const double* wide, uint8_t* out32);

/* Screen-space LOD selection of the forest generator, selectLOD
 * (raytracer/src/filtering/generate_random_forest.py:179-225), one tree after
 * the other in double precision (forest_oracle.c).  The two structs have the
 * layouts of the library's r2_lod_camera and r2_lod_volume. */
typedef struct orc_lod_camera {
  double world_to_view[16];
  double pos[3];
  double near_plane_distance, pixel_size, pixel_area;
  double sensor_width, sensor_height;
  double far_scale;
} orc_lod_camera;
typedef struct orc_lod_volume {
  double voxel_size;
  double bb_min[3], bb_max[3];
  double num_voxels[3];
  double corners[8][3];
} orc_lod_volume;
/* lod_out: index into lods or -1 (the mesh); also the inputs of the decision
 * per tree when diag is non-null: 3 doubles (covered pixels, -1 when all
 * corners are outside; the coarsest LOD's projected hull area; 0). */
int orc_select_lods(const orc_lod_camera* cam, const orc_lod_volume* lods, const uint32_t* model_first,
                    const uint32_t* model_count, uint32_t nmodels, const double* tree_pos, const double* tree_scaling,
                    const uint32_t* tree_model, uint32_t ntrees, double min_lod, double covered_pixels,
                    int32_t* lod_out, double* diag);

#ifdef __cplusplus
}
#endif
#endif
