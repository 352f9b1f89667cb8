/*
 * klon3d_mesh.h — C ABI of the body mesh as a signed-distance collider on
 * the device.
 *
 * This replaces the queries of `Koerpernetz` (viktoschi/GarmentCraft,
 * crates/klon3d-sim/src/netzkoerper.rs): the exact nearest point on the
 * surface signed by angle-weighted pseudonormals, and the segment
 * penetration test, each for a batch of points or segments. It adds what
 * the reference does not have: the voxelisation of the mesh into the sampled
 * grid that a K3D_BODY_SDF_GRID body (klon3d_step.h) reads, built from the
 * same exact query.
 *
 * Paths are relative to the reference project; `sim/` stands for
 * `crates/klon3d-sim/`. Plain pointers and sizes; every array is a host
 * array owned by the caller; the handle owns its device buffers and one CUDA
 * stream, and each call returns when its results are in the caller's arrays.
 * One handle is used by one thread at a time; each call makes the handle's
 * device current on the calling thread (as the solver's calls do).
 */
#ifndef KLON3D_MESH_H
#define KLON3D_MESH_H

#include <stdint.h>

#include "klon3d_step.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct k3d_mesh k3d_mesh;

/* Region of a nearest point (Region, sim/src/netzkoerper.rs:50-57): corner k
 * (0-2), edge k from corner k to k+1 (3-5), face (6); -1 = no hit. */
enum {
  K3D_REGION_ECKE0 = 0,
  K3D_REGION_KANTE0 = 3,
  K3D_REGION_FLAECHE = 6,
  K3D_REGION_KEINE = -1
};

/* Koerpernetz::neu (sim/src/netzkoerper.rs:297-367): punkte 3 per point (m,
 * z up), dreiecke 3 per triangle, counter-clockwise seen from outside. Refuses
 * (K3D_BAD_ARGUMENT, *out null, the reason in err when err_cap > 0) what the
 * reference refuses: no triangles, suchtiefe <= 0, an index out of range, an
 * edge with more than two triangles, two triangles running an edge the same
 * way, a volume <= 0. Open edges are allowed and counted. suchtiefe is the
 * search depth (SUCHTIEFE = 0.01 m, :46); the triangle grid has cells of
 * 2 * suchtiefe over the point hull grown by suchtiefe (:820-858). */
k3d_status k3d_mesh_create(const double* punkte, int64_t n_punkte, const uint32_t* dreiecke, int64_t n_dreiecke,
                           double suchtiefe, int32_t device, k3d_mesh** out, char* err, int64_t err_cap);
void k3d_mesh_destroy(k3d_mesh* m);
const char* k3d_mesh_last_error(const k3d_mesh* m);

/* Koerpernetz::nachfuehren (:390-411): new positions, same count and order;
 * normals, spheres, volume and the grid's cells are recomputed, the grid
 * grows with the body and never shrinks. K3D_BAD_ARGUMENT when the volume
 * turns <= 0 (the mesh keeps its previous positions then). */
k3d_status k3d_mesh_update(k3d_mesh* m, const double* punkte);

typedef struct k3d_mesh_info {
  int64_t n_punkte, n_dreiecke;
  int64_t randkanten;          /* open edges */
  double volumen;              /* m^3, summed on the device (tree order) */
  double suchtiefe;
  double gitter_ursprung[3];   /* triangle grid (Gitter, :75-142) */
  double gitter_zelle;
  int64_t gitter_zahl[3];
  int64_t gitter_eintraege;
  double ms_letzter_aufruf;    /* device time of the last query, update or voxelisation (CUDA events) */
  int64_t kernels_letzter_aufruf;
  int64_t ungeklaert;          /* voxelisation: nodes beyond the band whose sign the line passes left open */
} k3d_mesh_info;
k3d_status k3d_mesh_get_info(const k3d_mesh* m, k3d_mesh_info* out);

/* setze_punktgeschwindigkeit (:454-463): v 3 per point (m/s), the velocity
 * field of a deforming body, or null to clear it (the body moves rigidly
 * again). Contacts and the step's segment check then take the body's
 * velocity at the hit from the field (geschwindigkeit_an, :474-489, the
 * barycentric mix of the hit triangle's point velocities); k3d_mesh_update
 * clears the field, as nachfuehren does (:409). */
k3d_status k3d_mesh_set_velocity(k3d_mesh* m, const double* v);

/* geschwindigkeit_an (:474-489) per (triangle, point on it): out 3 per
 * point, starr (3) where no field is set. */
k3d_status k3d_mesh_velocity_at(k3d_mesh* m, const int32_t* dreieck, const double* punkt, int64_t n,
                                const double starr[3], double* out);

/* The point-dependent tables (punktabhaengig, :257-290) and the edge
 * neighbours (:319-337); any pointer may be null. flaechennormale 3 per
 * triangle, punktnormale 3 per point (angle-weighted, summed in triangle
 * order), nachbar 3 per triangle (the triangle itself at an open edge),
 * kugel 4 per triangle (bounding sphere centre, radius). */
k3d_status k3d_mesh_tables(k3d_mesh* m, double* flaechennormale, double* punktnormale, uint32_t* nachbar,
                           double* kugel);

/* Nearest surface point per query point x (3 per point).
 * radius > 0: Koerpernetz::naechster(x, radius) (:503-539), region and
 *   dreieck -1 where no surface point is closer than radius;
 * radius <= 0: Koerpernetz::naechster_alle (:770-782), over every triangle.
 * abstand is signed (outside positive, the pseudonormal's side, :492-499),
 * normale points outwards (the pseudonormal where the point is on the
 * surface). Among triangles at exactly the same distance the one the
 * reference keeps wins: the first in its cell order (radius > 0) or the
 * smallest index (radius <= 0). Any output pointer may be null. */
k3d_status k3d_mesh_nearest(k3d_mesh* m, const double* x, int64_t n, double radius, double* abstand, double* punkt,
                            double* normale, int32_t* dreieck, int32_t* region);

/* Koerpernetz::durchstoss (:541-593) per segment a -> b (3 per segment), in
 * the mesh's frame:
 * the first entry through the surface from outside (triangles facing the
 * segment's direction are skipped); dreieck -1 where there is none; punkt on
 * the segment, normale the triangle's face normal. Among entries at exactly
 * the same segment parameter the first in the reference's cell order wins. The body
 * velocity at the hit is k3d_mesh_velocity_at of (dreieck, punkt). */
k3d_status k3d_mesh_penetration(k3d_mesh* m, const double* a, const double* b, int64_t n, int32_t* dreieck,
                                double* punkt, double* normale);

/* The signed-distance grid of the mesh for a K3D_BODY_SDF_GRID body: node
 * (i, j, k) at ursprung + spacing * (i, j, k) in the mesh's frame (put the
 * mesh's offset into k3d_body.punkt and this ursprung into k3d_body.ursprung);
 * sdf receives dims[0] * dims[1] * dims[2] floats, x fastest.
 * band <= 0: every node holds the signed distance of naechster_alle.
 * band > 0 (band > spacing): a node closer to the surface than band holds its
 *   exact signed distance, every other node +-band with the sign of its
 *   connected region of such nodes, carried along grid lines from the band
 *   (for a closed mesh this is the pseudonormal's sign; a node whose sign no
 *   line reaches takes the exact query). */
k3d_status k3d_mesh_sdf(k3d_mesh* m, const int32_t dims[3], const double ursprung[3], double spacing, double band,
                        float* sdf);

#ifdef __cplusplus
}
#endif

#endif /* KLON3D_MESH_H */
