/*
 * klon3d_step.h — C ABI of the B200 implicit cloth step.
 *
 * This is the drop-in boundary for klon3d-sim's implicit backward-Euler step
 * (viktoschi/GarmentCraft, crates/klon3d-sim). A caller that today holds a
 * `Szene` and an `ImplizitCg` (implizit.rs:570-626) with a `Loeser` backend
 * (implizit.rs:304-351) binds these entry points instead. Plain pointers and
 * sizes only; the caller owns every host array, the solver handle owns its
 * device buffers. No call allocates device memory after k3d_upload_scene.
 *
 * Paths below are relative to the reference project; `sim/` stands for
 * `crates/klon3d-sim/`.
 *
 * Threading: one handle is used by one thread at a time (it owns one CUDA
 * stream); several handles may run on several threads.
 */
#ifndef KLON3D_STEP_H
#define KLON3D_STEP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define K3D_ABI_VERSION 4

/* Status of a call. Unconverged CG is data (k3d_cg_result), not an error,
 * as in CgLauf (sim/src/implizit.rs:294-299). */
typedef enum k3d_status {
  K3D_OK = 0,
  K3D_NOT_CONVERGED = 1, /* informational: a solve hit cg_max */
  K3D_BREAKDOWN = 2,     /* p^T A p <= DBL_MIN or not finite (implizit.rs:406-408) */
  K3D_NON_FINITE = 3,    /* a non-finite position or velocity after the step */
  K3D_DEVICE_ERROR = 4,  /* a CUDA call failed; see k3d_last_error */
  K3D_BAD_ARGUMENT = 5,  /* null pointer, size mismatch, index out of range */
  K3D_TIMEOUT = 6        /* a bounded device wait gave up (never expected) */
} k3d_status;

/* Arithmetic of the device step. FP64 mirrors the reference CPU solver;
 * MIXED evaluates forces, Hessian products and the preconditioner in FP32 and
 * keeps dot products, CG scalars, convergence test, dv and x/v in FP64.
 * MIXED_STORAGE stores the assembled operator blocks and the preconditioner in
 * FP32 (half the bytes the CG streams per iteration) and keeps the CG vectors
 * and their arithmetic in FP64: the CG then runs in FP64 on the FP32-rounded
 * operator, with the FP64 form's iteration counts. */
typedef enum k3d_precision { K3D_FP64 = 0, K3D_MIXED = 1, K3D_MIXED_STORAGE = 2 } k3d_precision;

/* ImplizitParameter (sim/src/implizit.rs:457-531), same meaning and defaults
 * (k3d_params_default). */
typedef struct k3d_params {
  int32_t schritte_je_bild;     /* substeps per frame, default 5 */
  int32_t cg_max;               /* CG iteration cap, default 50 */
  double cg_toleranz;           /* relative tolerance in the P^-1 norm, default 1e-5 */
  double naht_k;                /* seam spring N/m, default 500 */
  double kontakt_rand;          /* contact margin m, default 1e-4 */
  int32_t normalkraft_aus_last; /* friction normal force from the load, default 0 */
  int32_t durchstoss_pruefen;   /* segment-through-skin check (mesh bodies only), default 1 */
  int32_t selbstkollision;      /* cloth-cloth proximity springs (selbstkollision.rs:387-788), default 0 */
  int32_t precision;            /* k3d_precision, default K3D_FP64 */
  double selbst_zusatzdicke;    /* default 2.5e-3 m */
  double selbst_steifigkeit;    /* default 1e-3 */
  int32_t selbst_stoss_iterationen;   /* impact response passes (implizit.rs:491), default 1 */
  int32_t selbst_schnitte_an_naehten; /* edges through their seam partners' triangles count (:494), default 0 */
  int32_t koerperpunkt_durchgaenge;   /* body points against cloth triangles: passes per step (implizit.rs:479), default 0 = off */
  int32_t pcg_bloecke;                /* no reference counterpart: CTAs of the persistent PCG launch, at most one
                                         per SM times the CTAs that fit; 0 (default) = that maximum. Fewer CTAs
                                         make each grid barrier cheaper, which pays on small drapes */
  double koerperpunkt_tiefe;          /* m below a body point a triangle is still lifted (implizit.rs:481), default 0.01 */
  int32_t graph;                      /* no reference counterpart: 1 = each frame's launches are captured once as a
                                         CUDA graph and replayed while their arguments stay the same (recaptured
                                         when they change, e.g. a moving body); not with self-collision, whose
                                         stage reads counts back between launches. The per-frame PCG time of
                                         k3d_last_solve_ms stays 0 then. Default 0 */
  int32_t pcg_threads;                /* no reference counterpart: threads per CTA of the persistent PCG launch,
                                         256 (two CTAs per SM), 512 or 1024 (one per SM); 0 (default) = 512 */
} k3d_params;

/* Simparameter (sim/src/szene.rs:96-126), the part the implicit step reads. */
typedef struct k3d_simparams {
  double bild_dt;        /* frame length s, default 1/60 */
  double schwerkraft[3]; /* m/s^2, default (0, 0, -9.81) */
  double daempfung;      /* air damping 1/s, default 0 */
} k3d_simparams;

/* Body kinds. K3D_BODY_CYLINDER is Koerper::Zylinder (sim/src/koerper.rs:19).
 * K3D_BODY_SDF_GRID is a sampled signed-distance grid with trilinear value
 * and gradient (k3d_mesh_sdf in klon3d_mesh.h samples a body mesh into one).
 * K3D_BODY_MESH is Koerper::Netz (koerper.rs:20-24): a k3d_mesh (klon3d_mesh.h)
 * on the solver's device at offset `punkt`, moving rigidly with
 * `geschwindigkeit`; its contact is the exact nearest query within
 * max(search depth, distance) (koerper.rs:80-87), and the step's segment
 * check (k3d_params.durchstoss_pruefen, implizit.rs:988-1002) tests the
 * points' paths against it. The mesh must outlive the solver's use of it;
 * k3d_mesh_update between frames moves it. */
enum { K3D_BODY_CYLINDER = 0, K3D_BODY_SDF_GRID = 1, K3D_BODY_MESH = 2 };

struct k3d_mesh;

typedef struct k3d_body {
  int32_t art;              /* K3D_BODY_* */
  int32_t dims[3];          /* grid nodes along x, y, z (SDF grid) */
  double punkt[3];          /* cylinder: point on the axis; grid: offset of the grid */
  double achse[3];          /* cylinder axis (normalised on use) */
  double radius;            /* cylinder radius m */
  double geschwindigkeit[3];/* body velocity m/s; the body moves by v*t within a frame */
  double ursprung[3];       /* grid: position of node (0,0,0) relative to punkt */
  double spacing;           /* grid: node spacing m */
  const float* sdf;         /* grid: dims[0]*dims[1]*dims[2] values, x fastest (host) */
  int32_t instanz;          /* the instance it acts on in a batch scene, -1 = every instance */
  int32_t pad;
  const struct k3d_mesh* netz; /* K3D_BODY_MESH: the mesh (null otherwise) */
} k3d_body;

/* Szene (sim/src/szene.rs:198-269): the arrays the implicit step reads or
 * writes. Counts are element counts; index arrays are flattened rows. The
 * groups are in the scene's colour order. x and v are read and written by
 * k3d_frame; everything else is read only. */
typedef struct k3d_scene {
  int64_t n_punkte;
  double* x;                      /* 3 per point, m */
  double* v;                      /* 3 per point, m/s */
  const double* masse;            /* kg */
  const double* w;                /* inverse mass, 0 = pinned */
  const double* kollisionsabstand;/* half thickness m */
  const double* reibung;          /* friction coefficient */
  int64_t n_abstand;              /* distance constraints (Szene::abstand) */
  const uint32_t* abstand_punkte; /* 2 per constraint */
  const double* abstand_ruhe;
  const double* abstand_nachgiebigkeit;
  const uint8_t* membran_kante;   /* 1: carried by a membrane, k = 0 */
  int64_t n_naht;                 /* seam springs (Szene::naht) */
  const uint32_t* naht_punkte;    /* 2 per seam */
  const double* naht_ruhe;        /* rest length; +inf = open (current length) */
  int64_t n_biegung;              /* dihedral bending constraints */
  const uint32_t* biegung_punkte; /* 4 per constraint: edge i, j, then the two opposite points */
  const double* biegung_ruhe;
  const double* biegung_nachgiebigkeit;
  int64_t n_membran;              /* membrane elements (Szene::membran_elemente) */
  const uint32_t* membran_punkte; /* 3 per element */
  const double* membran_flaeche;  /* rest area m^2 */
  const double* membran_ruhe_inv; /* 4 per element, row-wise D^-1 */
  const double* membran_kette;    /* 2 per element: warp direction */
  const double* membran_schuss;   /* 2 per element: weft direction */
  const double* membran_steif;    /* 3 per element: E_warp, E_weft, G in N/m */
  int64_t n_dreiecke;             /* pattern triangles (Szene::dreiecke) */
  const uint32_t* dreiecke;       /* 3 per triangle */
  const double* ruhe_inv;         /* 4 per triangle */
  int32_t n_koerper;
  int32_t pad0;
  const k3d_body* koerper;
  k3d_simparams param;
  double zeit;
  /* Teilinfo (sim/src/szene.rs:181-194), read by self-collision only
   * (selbstkollision.rs:623-688). n_teile = 0 with null arrays: no parts
   * (every point and triangle gets stretch stiffness 0, no folded bands). */
  int64_t n_teile;
  const int64_t* teil_bereiche;  /* 4 per part: first point, end point, first triangle, end triangle */
  const double* teil_dehnung;    /* per part: the material's dehnung_n_m, N/m */
  const int32_t* teil_band_von;  /* per part: carrier part of a folded allowance band, -1 = none; may be null */
  /* Batch of independent drapes (no counterpart in the reference, which steps
   * one scene at a time). n_instanzen <= 1: one drape. Otherwise instance k
   * owns points [instanz_punkte[k], instanz_punkte[k + 1]); every element
   * lies within one instance, and each element group (abstand, naht, biegung,
   * membran) lists its elements instance by instance. The instances share one
   * PCG launch, each with its own blocks, reductions and convergence; bodies
   * act on the instance named in k3d_body.instanz. */
  int64_t n_instanzen;
  const int64_t* instanz_punkte;  /* n_instanzen + 1 point offsets, ascending from 0 to n_punkte */
} k3d_scene;

/* ImplizitStatistik (sim/src/implizit.rs:535-561), field for field. */
typedef struct k3d_stats {
  int64_t cg_iterationen;
  int64_t loesungen;
  int64_t nicht_konvergiert;
  int64_t kontakte;
  int64_t haftend;
  int64_t freigegeben;
  int64_t durchstoesse;
  int64_t koerperpunkte;
  double rest_max;
  int64_t naehe_punkt_dreieck;
  int64_t naehe_kante_kante;
  int64_t selbst_stoesse;
  int64_t durchdringungen;
  int64_t durchdringungsgebiete;
  /* not in ImplizitStatistik: solves that stopped on the CG breakdown guard
   * (implizit.rs:406-408), and the largest |dv| component of the frame's solves */
  int64_t zusammenbrueche;
  double dv_max;
} k3d_stats;

/* CgLauf (sim/src/implizit.rs:294-299). */
typedef struct k3d_cg_result {
  int64_t iterationen;
  int32_t nicht_konvergiert;
  int32_t breakdown;
  double rest;
} k3d_cg_result;

/* Readback of the system one substep would solve, the mirror of the
 * device-built system (GpuAufbau, sim/src/gpu.rs:1040-1065). Every pointer is
 * caller-owned and may be null to skip that field. */
typedef struct k3d_system_readback {
  double* rhs;      /* 3 per point, b = h (f - h H v) */
  double* f;        /* 3 per point, forces */
  double* last;     /* 3 per point, tension-only load plus weight */
  double* pinv;     /* 9 per point, inverse diagonal block of A, row-wise */
  double* normale;  /* 3 per point, contact normal, zero where not held */
  double* vn_soll;  /* 1 per point, required normal velocity (held points) */
  uint8_t* fest;    /* 1 per point, 1 = held */
} k3d_system_readback;

/* Pattern input of the scene builder: the part of klon3d_mesh::Musternetz
 * (crates/klon3d-mesh/src/lib.rs:91-241) that Szene::bauen reads. */
typedef struct k3d_material {
  double dehnung_n_m, kette_n_m, schub_n_m;
  double biegung_nm, biegung_kette_nm, biegung_schraege_nm;
  double flaechengewicht_kg_m2, dicke_m, reibung;
} k3d_material;

typedef struct k3d_piece {
  int64_t n_punkte;
  const double* punkte_mm;  /* 2 per point, pattern coordinates (mm) */
  int64_t n_dreiecke;
  const uint32_t* dreiecke; /* 3 per triangle, positive orientation */
  double fadenlauf[2];      /* grainline in pattern coordinates */
  k3d_material material;
  double reduktion;
  const double* lage;       /* 3 per point: start position (m) */
} k3d_piece;

typedef struct k3d_seam_part {
  int32_t teil_a, teil_b;
  int64_t n_paare;
  const uint32_t* paare; /* 2 per pair: local point on piece a, on piece b */
} k3d_seam_part;

typedef struct k3d_seam {
  int32_t n_teilnaehte;
  int32_t pad0;
  const k3d_seam_part* teilnaehte;
  double laenge_a_mm, laenge_b_mm;
} k3d_seam;

typedef struct k3d_pattern {
  int32_t n_teile;
  int32_t n_naehte;
  const k3d_piece* teile;
  const k3d_seam* naehte;
  k3d_simparams param;
  double naht_nachgiebigkeit;
  int32_t einhalteweite;
  int32_t pad0;
} k3d_pattern;

typedef struct k3d_solver k3d_solver;
typedef struct k3d_built_scene k3d_built_scene;

/* ---------------------------------------------------------------- library */
int32_t k3d_abi_version(void);
void k3d_params_default(k3d_params* out);            /* ImplizitParameter::default, implizit.rs:505-531 */
void k3d_simparams_default(k3d_simparams* out);      /* Simparameter::default, szene.rs:115-126 */

/* ---------------------------------------------------------------- scene builder
 * Szene::aus_netz (sim/src/szene.rs:284-292, 320-715) for a pattern given as
 * pieces and seam point pairs, without the folded allowance band. The built
 * scene owns its arrays; k3d_built_scene_view fills `out` with pointers into
 * them (valid until k3d_built_scene_free). */
k3d_status k3d_build_scene(const k3d_pattern* pattern, k3d_built_scene** out);
k3d_status k3d_built_scene_view(k3d_built_scene* built, k3d_scene* out);
void k3d_built_scene_free(k3d_built_scene* built);

/* ---------------------------------------------------------------- solver
 * ImplizitCg::mit_loeser (implizit.rs:615-626) with the device backend. */
k3d_solver* k3d_solver_create(const k3d_params* params, int32_t device);
void k3d_solver_destroy(k3d_solver* h);
const char* k3d_last_error(const k3d_solver* h);
/* Loeser::name (implizit.rs:306), e.g. "B200 (f64)". */
const char* k3d_solver_name(const k3d_solver* h);

/* Uploads topology, material, bodies and state. Replaces the topology upload
 * of GpuLoeser::hochladen (gpu.rs:1428-1456); call again when the topology,
 * the bodies or the rest lengths change. Resets the CG warm start. */
k3d_status k3d_upload_scene(k3d_solver* h, const k3d_scene* s);

/* Rechenweg::bild (sim/src/cpu.rs:58-60, implizit.rs:1042-1057): one frame of
 * schritte_je_bild substeps. Uploads s->x and s->v, runs the frame on the
 * device, writes s->x, s->v back and advances s->zeit. `stats` may be null. */
k3d_status k3d_frame(k3d_solver* h, k3d_scene* s, k3d_stats* stats);

/* The same frame on the device-resident state (no host copies), `n_frames`
 * times. State moves in and out with k3d_upload_state / k3d_download_state. */
k3d_status k3d_frames_resident(k3d_solver* h, int32_t n_frames, k3d_stats* stats);
k3d_status k3d_upload_state(k3d_solver* h, const double* x, const double* v);
k3d_status k3d_download_state(k3d_solver* h, double* x, double* v);

/* ImplizitCg::operator (implizit.rs:637-643): builds the system of the next
 * substep at the scene's current state (uploaded x, v) and applies A to p. */
k3d_status k3d_operator(k3d_solver* h, const double* p, double* out);

/* ImplizitCg::system_fuer (implizit.rs:651-654) as a readback of the
 * device-built system (the fields of GpuAufbau, gpu.rs:1040-1065). */
k3d_status k3d_system_for(k3d_solver* h, k3d_system_readback* out);

/* Loeser::loese (implizit.rs:308, 370-426) on the device-built system of the
 * current state, with the contact set of that state. dv_inout is the warm
 * start in and the solution out (3 per point). */
k3d_status k3d_solve(k3d_solver* h, double* dv_inout, k3d_cg_result* out);

/* The contact set Loeser::loese receives (`fest: &[Option<Fest>]`,
 * implizit.rs:308; Fest at :594-599) as arrays over the points: fest[i] = 1
 * holds point i (Some) with the unit normal normale[3i..3i+2] and the normal
 * velocity vn_soll[i] it must have after the step; fest[i] = 0 leaves it
 * free (None). Fest::v_koerper is not read by a solve. Host pointers. */
typedef struct k3d_contact_set {
  const uint8_t* fest;
  const double* normale;
  const double* vn_soll;
} k3d_contact_set;

/* Loeser::loese (implizit.rs:308) with the caller's contact set, as
 * ImplizitCg::schritt hands its host-built set to every backend
 * (implizit.rs:870-883), one that builds the system itself included
 * (GpuLoeser::loese, gpu.rs:1808-1817): the device builds the system of the
 * current state and solves it with `fest` in place of the contact set it
 * would find against the bodies. dv_inout as in k3d_solve. */
k3d_status k3d_solve_contacts(k3d_solver* h, const k3d_contact_set* fest, double* dv_inout, k3d_cg_result* out);

/* Loeser::rest_geloest (implizit.rs:337-342): A dv - b without the filter. */
k3d_status k3d_residual(k3d_solver* h, const double* dv, double* out);

/* Loeser::last_lesen (implizit.rs:348-350): the load of the last built system. */
k3d_status k3d_read_load(k3d_solver* h, double* out);

/* The CG warm start the next substep starts from (ImplizitCg's private
 * dv_vorher, implizit.rs:578, 906, 945): the last solve's dv, 3 per point,
 * which k3d_frame and k3d_frames_resident carry from substep to substep. The
 * reference has no accessor for it; with it a caller can hand the device's
 * state, warm start included, to another solver (e.g. a CPU cross-check). */
k3d_status k3d_read_warm_start(k3d_solver* h, double* dv);

/* Time of the last device frame in ms, measured with CUDA events on the
 * handle's stream (the figure GpuLoeser::zeiten reports, gpu.rs:1225-1227). */
double k3d_last_frame_ms(const k3d_solver* h);

/* Time of the PCG launches (solve and release test) of the last frame call,
 * in ms, CUDA events on the handle's stream around each of them. */
double k3d_last_solve_ms(const k3d_solver* h);

/* Number of device kernels the handle launched since creation. */
int64_t k3d_kernel_launches(const k3d_solver* h);

/* No reference counterpart: CTAs of the handle's persistent PCG launch
 * (k3d_params.pcg_bloecke, capped at the most that can be resident at once);
 * 0 when the handle has no device. */
int32_t k3d_pcg_blocks(const k3d_solver* h);

/* ---------------------------------------------------------------- adjoint
 * The reference has no differentiation; these have no counterpart in it.
 * They differentiate the step k3d_frames_resident takes, with its discrete
 * decisions as the forward took them (the contact set after the release
 * pass, stick or slip, which bodies pushed a point out). They need
 * K3D_FP64, self-collision off, normalkraft_aus_last off and at most 14
 * bodies (K3D_BAD_ARGUMENT otherwise). */
typedef struct k3d_adjoint_stats {
  int64_t cg_iterationen;    /* adjoint PCG iterations, all substeps */
  int64_t loesungen;
  int64_t nicht_konvergiert;
  int64_t zusammenbrueche;
  double ms_vorwaerts;       /* device time of the last k3d_adjoint_forward */
  double ms_rueckwaerts;     /* device time of k3d_adjoint_backward, recomputation included */
  double ms_neuberechnung;   /* the recomputation of the segments within it */
} k3d_adjoint_stats;

/* n_frames frames on the device-resident state, as k3d_frames_resident, that
 * keep x, v and the warm start on the device every k substeps. */
k3d_status k3d_adjoint_forward(k3d_solver* h, int32_t n_frames, int32_t k, k3d_stats* stats);

/* The adjoint of the frames of the last k3d_adjoint_forward. gx, gv: the
 * cotangents of the final x, v (host, 3 per point). Writes, where the
 * pointer is not null, the cotangents of the initial x and v (3 per point),
 * per membrane those of (E_warp, E_weft, G, a rotation of its grain basis in
 * the rest plane) (4 per membrane, the scene's membrane order) and per hinge
 * that of its stiffness k = 1/biegung_nachgiebigkeit, summed over the
 * substeps. Each segment of k substeps is computed again from its checkpoint;
 * afterwards the resident state is the forward's final state. */
k3d_status k3d_adjoint_backward(k3d_solver* h, const double* gx, const double* gv, double* gx0, double* gv0,
                                double* g_membran, double* g_biegung, k3d_adjoint_stats* stats);

/* ---------------------------------------------------------------- no allocation
 * k3d_operator_noalloc has no counterpart in the reference. It is A p as
 * k3d_operator computes it (FP64, the scene's positions s->x), for a caller
 * that must not allocate device memory: a host application or framework that
 * owns the whole device memory budget through its own pool and forbids
 * cudaMalloc/cudaFree behind its back, or a real-time loop that must never
 * block in the driver's allocator. No handle is needed and nothing is
 * allocated: every pointer in `s` (x, masse and the constraint arrays; v, w,
 * bodies are not read) and `p`, `out` (3 doubles per point) are DEVICE
 * pointers owned by the caller, and the only scratch is a static array of
 * 3 MiB inside the library, present on every GPU that loads it until the
 * process exits. Limits: s->n_punkte <= 131072 (K3D_BAD_ARGUMENT beyond);
 * params->selbstkollision must be 0 (the proximity springs belong to a
 * handle's self-collision stage; K3D_BAD_ARGUMENT otherwise). A non-finite
 * position, mass or p gives NaN in `out` and K3D_NON_FINITE. The first call
 * on a device looks the scratch up for that device; make that first call
 * before any stream capture. Calls share the scratch, so calls that overlap
 * on the GPU (other streams, other host threads) race; the call clears what
 * it needs and synchronises `stream` (a cudaStream_t, null = the legacy
 * default stream) before it returns. An element that names a point out of
 * range is skipped and reported as K3D_BAD_ARGUMENT. */
k3d_status k3d_operator_noalloc(const k3d_params* params, const k3d_scene* s, const double* p, double* out,
                                void* stream);

/* ---- self-collision probes (proximity stage, sim/src/selbstkollision.rs)
 * Readbacks of the stage's last run, which every frame, operator, system,
 * solve and residual call makes first when k3d_params.selbstkollision is set
 * (the penetration and impact stages of the reference are not part of it).
 * Each returns -1 when self-collision is off or has not run (k3d_last_error
 * says which); otherwise the full count, filling at most `cap` entries of
 * every non-null array. */

/* selbstkollision::finde (:387-398): the proximity pairs in the reference's
 * order (point-triangle pairs by triangle, then edge-edge pairs by edge).
 * art: 0 point-triangle, 1 edge-edge; punkte and gewichte 4 per pair (the
 * weighted sum of the points is the gap vector from the second side to the
 * first); normale 3 per pair; abstand; ruhe (the rest distance as found). */
int64_t k3d_selfcollision_pairs(k3d_solver* h, int64_t cap, int32_t* art, uint32_t* punkte, double* gewichte,
                                double* normale, double* abstand, double* ruhe);

/* Hashgitter (:256-345) of the point boxes (kanten = 0) or the edge boxes
 * (kanten = 1): returns the bucket count; anfang receives the bucket starts
 * (bucket count + 1 values), eintraege the entries, *n_eintraege their count. */
int64_t k3d_selfcollision_hash(k3d_solver* h, int32_t kanten, int64_t cap_anfang, uint32_t* anfang,
                               int64_t cap_eintraege, uint32_t* eintraege, int64_t* n_eintraege);

/* selbstkollision::federn (:713-787): per pair the force on the first side
 * (3 values) and the 3x3 block k[(1 - mu) n n^T + mu I] (9 values, row-major). */
int64_t k3d_selfcollision_springs(k3d_solver* h, int64_t cap, double* kraft, double* block);

#ifdef __cplusplus
}
#endif
#endif /* KLON3D_STEP_H */
