/*
 * prr_oracle.h -- test infrastructure only (the oracle).
 *
 * A plain-C CPU restatement of the reference renderer's closest-hit path and
 * of the small numeric kernels around it. Only tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py load it, as the checker; the product
 * never links it. Every function cites the reference file:line it restates.
 *
 * Pinned against the reference itself: tests/golden/ holds fixtures made by
 * running the reference sources (oracle/_ref/libprr_ref.so, IEEE build) and
 * tests/test_oracle.py checks this restatement against them bit for bit.
 */
#ifndef PRR_ORACLE_H
#define PRR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- counter-keyed SplitMix64 (replaces global.hpp:35-50) ---- */
uint64_t prr_oracle_path_state(uint64_t seed, uint32_t stream, uint32_t index);
float prr_oracle_rand(uint64_t *state);
void prr_oracle_rng_stream(uint64_t seed, uint32_t stream, uint32_t index, int n, float *out);

/* ---- binned-SAH BVH over axis-aligned prim bounds (BVH.cpp:13-280) ----
 * prim_bounds: n x 6 floats (minx,miny,minz,maxx,maxy,maxz); prim_area: n.
 * Outputs sized by the caller: up to 2n-1 nodes. Returns the node count. */
int64_t prr_oracle_bvh_build(const float *prim_bounds, const float *prim_area, int64_t n,
                             int max_prims_in_node, float *node_bounds /* 6 per node */,
                             uint32_t *first_child, uint32_t *meta, float *node_area,
                             int32_t *ordered);

/* Triangle soup (n x 9 floats) -> prim bounds and areas as Triangle.hpp:30-36,
 * :183-185 compute them. */
void prr_oracle_triangle_prims(const float *verts, int64_t n, float *prim_bounds, float *area);

/* ---- closest hit / any hit on one triangle mesh (BVH.cpp:311-473,
 *      Triangle.hpp:46-92) ---- */
typedef struct prr_oracle_mesh prr_oracle_mesh;
prr_oracle_mesh *prr_oracle_mesh_new(const float *verts, int64_t ntri);
void prr_oracle_mesh_free(prr_oracle_mesh *m);
int64_t prr_oracle_mesh_nodes(const prr_oracle_mesh *m, float *bounds, uint32_t *first_child,
                              uint32_t *meta, float *areas, int32_t *ordered);
/* id: input-order triangle index or -1; t: fp32 closest t; t64: winner re-solved
 * in fp64 (NaN on miss); visits/tests: interior-node visits and triangle tests. */
void prr_oracle_mesh_intersect(const prr_oracle_mesh *m, const float *o, const float *d,
                               int64_t n, int32_t *id, float *t, double *t64, int32_t *visits,
                               int32_t *tests, int nthreads);
void prr_oracle_mesh_occluded(const prr_oracle_mesh *m, const float *o, const float *d,
                              const float *tmax, int64_t n, uint8_t *hit, int nthreads);

/* ---- display transform (Renderer.cpp:149-171, ToneMapping.hpp:45-279) ----
 * mapper 0 Raw, 1 Standard, 2 AgX, 3 PBRNeutral, 4 ACES (Narkowicz 2015 fit). */
void prr_oracle_tonemap(int mapper, float exposure, const float *in_rgb, int64_t n,
                        float *out_rgb, uint8_t *out_u8);

/* ---- environment map CDF (EnvMap.hpp:189-224) ---- */
void prr_oracle_env_cdf(const float *rgb, int w, int h, float *cdf, float *marginal,
                        float *total);

/* ---- photon grid + fixed-radius irradiance (Photon.cpp:24-94) ----
 * rec: n x 9 floats (position, direction, power). */
void prr_oracle_photon_estimate(const float *rec, int64_t n, float radius, const float *q,
                                int64_t nq, float *out_rgb, int32_t *grid_res);
/* The same with a k-nearest cap (k > 0; 0 = fixed radius); inside (optional)
 * gets the number of photons inside the radius of each query. */
void prr_oracle_photon_estimate_knn(const float *rec, int64_t n, float radius, int k,
                                    const float *q, int64_t nq, float *out, int32_t *inside,
                                    int32_t *grid_res);

#ifdef __cplusplus
}
#endif
#endif
