// ORACLE — test infrastructure only. A CPU FP64 restatement of klon3d-sim's
// implicit backward-Euler cloth step (crates/klon3d-sim, viktoschi/GarmentCraft).
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
// it, and only as the checker or the timed CPU baseline. The product library
// (garmentcraft_b200) never links or calls it.
//
// Parity is pinned by the reference's own known-answer tests, restated in
// tests/test_oracle_golden.py (bending stiffness values, dihedral gradient vs
// central differences, membrane acceptance items, 3x3 inverse, seam spring
// convergence, tube hoop strain). The reference is Rust and cannot be built
// in this environment, so no reference binary exists to compare against.
//
// Every function cites the reference file:line it follows. Paths are relative
// to the reference project; `sim/` stands for `crates/klon3d-sim/`.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <map>
#include <optional>
#include <set>
#include <string>
#include <utility>
#include <vector>

namespace orc {

using V3 = std::array<double, 3>;
using V2 = std::array<double, 2>;
using M3 = std::array<V3, 3>;

// sim/src/koerper.rs:37-54 vector helpers
inline V3 sub(V3 a, V3 b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline V3 add(V3 a, V3 b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline V3 mul(V3 a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
inline double dot(V3 a, V3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 cross(V3 a, V3 b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

// ---------------------------------------------------------------- material
// sim/src/material.rs:21-68
struct Material {
  double dehnung_n_m = 0, kette_n_m = 0, schub_n_m = 0;
  double biegung_nm = 0, biegung_kette_nm = 0, biegung_schraege_nm = 0;
  double flaechengewicht_kg_m2 = 0, dicke_m = 0, reibung = 0;
};

// ---------------------------------------------------------------- membrane
// sim/src/kontinuum.rs:70-88 (Membran), :117-127 (Hessen)
struct Membran {
  double flaeche = 0;
  std::array<double, 4> ruhe_inv{};
  V2 kette{}, schuss{};
  double kette_n_m = 0, dehnung_n_m = 0, schub_n_m = 0;
};
struct Hessen {
  V3 f1{}, f2{}, w{};
};
struct MembranElement {
  std::array<uint32_t, 3> punkte{};
  Membran element;
};

std::optional<Membran> membran_bauen(std::array<V2, 3> ruhe, V3 kanten, V2 dir2, V3 material);
void membran_f(const Membran& m, const std::array<V3, 3>& p, V3& f1, V3& f2);
V3 membran_dehnung(const Membran& m, const std::array<V3, 3>& p);
V3 membran_spannung(const Membran& m, const std::array<V3, 3>& p);
double membran_energie(const Membran& m, const std::array<V3, 3>& p);
std::array<V3, 3> membran_krafte(const Membran& m, const std::array<V3, 3>& p);
std::array<V3, 3> membran_krafte_zug(const Membran& m, const std::array<V3, 3>& p);
Hessen membran_hessen(const Membran& m, const std::array<V3, 3>& p);
// kontinuum.rs:526-551 (Zug): one scalar XPBD constraint of a membrane
struct Zug {
  double c = 0;
  std::array<V3, 3> grad{};
  double alpha = 0;
};
std::array<Zug, 3> membran_zuege(const Membran& m, const std::array<V3, 3>& p);
std::array<V3, 3> membran_mal_h_aus(const Membran& m, const Hessen& h, const std::array<V3, 3>& d);
std::array<M3, 3> membran_diag_bloecke_aus(const Membran& m, const Hessen& h);
V3 psd2(double a, double b, double c);

// ---------------------------------------------------------------- bending
// sim/src/biegung.rs:92-173
double steifigkeit(double weft, double warp, double bias, double theta);
double steifigkeit_aus(double c2, double s2, double weft, double warp, double bias);
bool cos2_sin2(V2 e, V2 warp, double& c2, double& s2);
// sim/src/cpu.rs:279-307
double winkel_fehler(double theta, double ruhe);
bool dieder(const std::array<V3, 4>& q, double& theta, std::array<V3, 4>& grad);

// ---------------------------------------------------------------- colouring
// sim/src/faerbung.rs:11-57
std::pair<std::vector<uint32_t>, size_t> faerbe(size_t anzahl, size_t npunkte,
                                                 const std::vector<std::vector<uint32_t>>& punkte);
std::pair<std::vector<size_t>, std::vector<std::pair<size_t, size_t>>> ordnung(
    const std::vector<uint32_t>& farbe, size_t zahl);

// ---------------------------------------------------------------- bodies
// sim/src/koerper.rs:16-35 (Zylinder, Netz) plus a sampled signed-distance
// grid, which has no counterpart in the reference.
struct Koerpernetz;
struct Kontakt {
  V3 normale{};
  double tiefe = 0;
  V3 geschwindigkeit{};
};
struct Koerper {
  int art = 0;  // 0 = Zylinder, 1 = SDF grid, 2 = Netz (punkt is its offset)
  V3 punkt{}, achse{0, 0, 1};
  double radius = 0;
  V3 geschwindigkeit{};
  // grid: node (i,j,k) sits at ursprung + spacing*(i,j,k) + punkt (punkt moves)
  const float* sdf = nullptr;
  std::array<int32_t, 3> dims{};
  V3 ursprung{};
  double spacing = 1;
  const Koerpernetz* netz = nullptr;  // art 2; owned by the caller
  std::optional<Kontakt> kontakt(V3 x, double abstand) const;
  // koerper.rs:99-107: entry point, face normal, body velocity at the entry
  std::optional<std::array<V3, 3>> durchstoss(V3 von, V3 nach) const;
  // koerper.rs:113-118: body points against cloth triangles (mesh only)
  size_t punkte_gegen_dreiecke(double tief, const std::vector<std::array<uint32_t, 3>>& dreiecke,
                               const std::vector<double>& w, std::vector<V3>& x, std::vector<V3>& v) const;
  Koerper verschoben(double t) const;
};

// ---------------------------------------------------------------- body mesh
// sim/src/netzkoerper.rs:49-175 (Region, Naechster, Gitter, Koerpernetz).
// Regions: 0-2 corner k, 3-5 edge k (corner k to k+1), 6 face.
struct Naechster {
  double abstand = 0;  // outside positive
  V3 punkt{}, normale{};
  uint32_t dreieck = 0;
  int region = 6;
};
struct Durchstoss {
  V3 punkt{}, normale{};
  uint32_t dreieck = 0;
};
struct NetzGitter {
  V3 ursprung{};
  double zelle = 0;
  std::array<size_t, 3> zahl{};
  std::vector<uint32_t> anfang, eintraege;
  std::array<int64_t, 3> index(V3 x) const;
  size_t zellnummer(size_t kx, size_t ky, size_t kz) const;
  bool bereich(V3 lo, V3 hi, std::array<std::pair<size_t, size_t>, 3>& r) const;
};
std::pair<V3, int> naechster_auf_dreieck(V3 p, V3 a, V3 b, V3 c);
struct Koerpernetz {
  std::vector<V3> punkte;
  std::vector<std::array<uint32_t, 3>> dreiecke;
  std::vector<V3> flaechennormale;
  std::vector<std::array<uint32_t, 3>> nachbar;
  std::vector<V3> punktnormale;
  std::vector<std::pair<V3, double>> kugel;
  double suchtiefe = 0;
  NetzGitter gitter;
  NetzGitter punktgitter;  // the same cells, entries the body points (netzkoerper.rs:863-879)
  size_t randkanten = 0;
  double volumen = 0;
  std::vector<V3> punktgeschwindigkeit;  // empty: the body moves rigidly
  std::optional<std::string> setze_punktgeschwindigkeit(const std::vector<V3>& v);
  V3 geschwindigkeit_an(size_t t, V3 p, V3 starr) const;
  static std::optional<std::string> neu(std::vector<V3> p, std::vector<std::array<uint32_t, 3>> d, double suchtiefe,
                                        Koerpernetz& out);
  std::optional<std::string> nachfuehren(const std::vector<V3>& p);
  V3 kantennormale(size_t t, int k) const;
  V3 pseudonormale(size_t t, int r) const;
  Naechster ergebnis(V3 x, size_t t, V3 c, int r) const;
  std::optional<Naechster> naechster(V3 x, double radius) const;
  Naechster naechster_alle(V3 x) const;
  std::optional<Durchstoss> durchstoss(V3 a, V3 b) const;
  void sdf(const int32_t dims[3], V3 ursprung, double spacing, double band, float* out) const;
  // netzkoerper.rs:612-690
  size_t punkte_gegen_dreiecke(double tief, V3 versatz, V3 geschwindigkeit,
                               const std::vector<std::array<uint32_t, 3>>& dreiecke, const std::vector<double>& w,
                               std::vector<V3>& x, std::vector<V3>& v) const;
  void gitter_bauen();
};

// ---------------------------------------------------------------- scene
// sim/src/szene.rs:96-126
struct Simparameter {
  double bild_dt = 1.0 / 60.0;
  V3 schwerkraft{0, 0, -9.81};
  double daempfung = 0.0;
  double naht_nachgiebigkeit = 0.0;
  bool einhalteweite = false;
};
// sim/src/szene.rs:130-179
template <int N>
struct Gruppe {
  std::vector<std::array<uint32_t, N>> punkte;
  std::vector<double> ruhe, nachgiebigkeit;
  std::vector<std::pair<size_t, size_t>> farben;
  size_t size() const { return punkte.size(); }
};
// sim/src/szene.rs:181-194 (Teilinfo: the fields self-collision reads)
struct Teilinfo {
  size_t p0 = 0, p1 = 0;  // point range
  size_t d0 = 0, d1 = 0;  // triangle range
  double dehnung_n_m = 0;
  int64_t band_von = -1;  // carrier part of a folded allowance band, -1 = none
};
// sim/src/szene.rs:198-269 (the fields the implicit step reads)
struct Szene {
  std::vector<V3> x, v;
  std::vector<double> masse, w, kollisionsabstand, reibung;
  Gruppe<2> abstand, naht;
  Gruppe<4> biegung;
  std::vector<std::array<uint32_t, 3>> dreiecke;
  std::vector<std::array<double, 4>> ruhe_inv;
  std::vector<uint8_t> membran_kante;
  std::vector<MembranElement> membran_elemente;
  std::vector<Koerper> koerper;
  std::vector<Teilinfo> teile;
  Simparameter param;
  double zeit = 0;
  size_t membran_entartet = 0, naht_biegung_ohne = 0, einhalte_kanten = 0;
};

// Pattern input of the scene builder: the part of klon3d_mesh::Musternetz
// (crates/klon3d-mesh/src/lib.rs:91-241) that Szene::bauen reads.
struct Teil {
  std::vector<V2> punkte_mm;
  std::vector<std::array<uint32_t, 3>> dreiecke;
  V2 fadenlauf{1, 0};
  Material material;
  double reduktion = 0;
  std::vector<V3> lage;  // start position per point (m)
};
struct Teilnaht {
  size_t teil_a = 0, teil_b = 0;
  std::vector<std::pair<uint32_t, uint32_t>> paare;
};
struct Naht {
  std::vector<Teilnaht> teilnaehte;
  double laenge_a_mm = 0, laenge_b_mm = 0;
};
struct Muster {
  std::vector<Teil> teile;
  std::vector<Naht> naehte;
};
Szene szene_bauen(const Muster& netz, const std::vector<Koerper>& koerper, Simparameter param);
void naht_kuerzen(Szene& s, double schritt);
void naht_offen(Szene& s);

// ---------------------------------------------------------------- implicit
// sim/src/implizit.rs:79-100
struct Kante {
  uint32_t i = 0, j = 0;
  double k = 0;
  V3 richtung{};
  double quer = 0, ruhe = 0;
};
struct Biegung {
  std::array<uint32_t, 4> punkte{};
  std::array<V3, 4> grad{};
  double k = 0, ruhe = 0;
};
// ---------------------------------------------------------------- self-collision
// sim/src/selbstkollision.rs:41-588 (proximity stage: search and springs)
constexpr double ZUSCHLAG_QUADER = 2e-5;
constexpr double ZUSCHLAG_PAAR = 4e-5;
constexpr double KANTE_MIN = 1e-4;
constexpr double AUSLENKUNG_MAX = 2.5e-3;
constexpr double ANNAEHERUNG_ANTEIL = 1.0 / 32.0;
constexpr uint32_t KEIN = 0xffffffffu;
using Quader = std::pair<V3, V3>;
enum class Art { PunktDreieck = 0, KanteKante = 1 };
struct Naehe {
  Art art = Art::PunktDreieck;
  std::array<uint32_t, 4> punkte{};
  std::array<double, 4> gewichte{};
  V3 normale{};
  double abstand = 0, ruhe = 0;
};
struct Stoffnetz {
  std::vector<std::array<uint32_t, 3>> dreiecke;
  std::vector<std::array<uint32_t, 2>> kanten, kanten_dreiecke;
  std::vector<std::array<uint32_t, 3>> dreieck_kanten;
  std::vector<double> r_punkt, r_kante, r_dreieck;
  std::map<std::pair<uint32_t, uint32_t>, uint32_t> kanten_index;
  std::vector<std::vector<uint32_t>> naht_partner;
  std::vector<uint32_t> teil_von, band_von;
  std::vector<double> dicke;
  bool band_und_traeger(uint32_t a, uint32_t b) const;
  std::optional<double> band_abstand(uint32_t a, const uint32_t* andere, int n) const;
  bool gleich_oder_partner(uint32_t a, uint32_t b) const;
};
Stoffnetz stoffnetz_neu(const std::vector<std::array<uint32_t, 3>>& dreiecke, std::vector<double> r_punkt);
struct Normalen {
  std::vector<V3> dreieck, punkt, kantenebene;
};
Normalen normalen_neu(const Stoffnetz& netz, const std::vector<V3>& x);
int64_t zellindex(double x, double zelle);
size_t streue(int64_t i, int64_t j, int64_t k, size_t n);
struct Hashgitter {
  double zelle = 0;
  size_t eimer = 0;
  std::vector<uint32_t> anfang, eintraege;
};
Hashgitter hashgitter_neu(const std::vector<Quader>& quader, double zelle);
Quader quader_punkte(const V3* p, int n, double m);
Quader kanten_quader(V3 a, V3 b, double m);
std::array<double, 3> naechster_dreieck(V3 p0, V3 p1, V3 p2, V3 x);
// the hash cell size of both searches (selbstkollision.rs:402,514)
double hash_zelle(const Stoffnetz& netz);
std::vector<Naehe> finde(const Stoffnetz& netz, const std::vector<V3>& x, const std::vector<double>& w, bool pd,
                         bool kk);
struct Stoffwerte {
  std::vector<double> e_punkt, a_punkt, e_kante, a_kante, e_dreieck, a_dreieck, mu_punkt;
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> naht_partner;
};
std::pair<Stoffnetz, Stoffwerte> aus_szene(const Szene& s, double zusatzdicke);
// sim/src/selbstkollision.rs:691-697
struct Feder {
  std::array<uint32_t, 5> punkte{};
  std::array<double, 5> gewichte{};
  V3 kraft{};
  M3 block{};
};
// selbstkollision.rs:810-826, 1092-1114: an edge through a triangle; an impact
struct Schnitt {
  uint32_t kante = 0, dreieck = 0;
  double t = 0;
  std::array<double, 3> w{};
  V3 richtung{};
  double gewicht = 0;
};
struct Stoss {
  Art art = Art::PunktDreieck;
  std::array<uint32_t, 4> punkte{};
  std::array<double, 2> lage{};
  double zeit = 0, seite = 0;
  V3 normale{};
};
constexpr double STOSS_ABSTAND = 1e-4, STOSS_KANTE_MIN = 1e-4, SCHUB_HEBEL = 1e-3;
constexpr uint32_t FOLGE_MAX = 5;
std::vector<Schnitt> finde_schnitte(const Stoffnetz& netz, const std::vector<V3>& x, bool an_naehten);
std::vector<size_t> gebiete(const Stoffnetz& netz, std::vector<Schnitt>& schnitte);
std::vector<Stoss> finde_stoesse(const Stoffnetz& netz, const std::vector<V3>& x0, const std::vector<V3>& x1,
                                 const std::vector<double>& w, bool pd, bool kk);
std::vector<Stoss> ohne_durchdrungene(const Stoffnetz& netz, std::vector<Stoss> stoesse,
                                      const std::vector<Schnitt>& schnitte);
size_t stossantwort(const std::vector<Stoss>& stoesse, std::vector<V3>& x, const std::vector<double>& masse,
                    const std::vector<double>& w, size_t iterationen);
std::vector<Feder> schubfedern(const Stoffnetz& netz, const Stoffwerte& werte, const std::vector<Schnitt>& schnitte,
                               const std::vector<size_t>& wurzeln, double steifigkeit, std::vector<uint32_t>& folge,
                               const std::function<bool(std::array<uint32_t, 2>, std::array<uint32_t, 3>)>& eingeklemmt);
std::vector<Feder> federn(const Stoffnetz& netz, const Stoffwerte& werte, const std::vector<Naehe>& naehe,
                          double steifigkeit, const std::vector<double>& masse, const std::vector<double>& w,
                          const std::vector<double>& naht_ruhe, std::vector<V3>& v);

// sim/src/implizit.rs:594-599
struct Fest {
  V3 normale{};
  double vn_soll = 0;
  V3 v_koerper{};
};
// sim/src/implizit.rs:124-172
struct System {
  double h = 0, c = 0;
  size_t cg_max = 0;
  double cg_toleranz = 0;
  const std::vector<double>* masse = nullptr;
  const std::vector<double>* w = nullptr;
  const std::vector<V3>* v = nullptr;
  std::vector<Kante> kanten, naehte;
  std::vector<Biegung> biegungen;
  const std::vector<MembranElement>* membran = nullptr;
  std::vector<Hessen> membran_h;
  std::vector<Feder> federn;
  std::vector<V3> rhs, f, last;
  std::vector<M3> pinv;
  void mal_h(const std::vector<V3>& p, std::vector<V3>& out) const;
  void mal_a(const std::vector<V3>& p, std::vector<V3>& out) const;
  std::vector<M3> diag() const;
};
// sim/src/implizit.rs:294-299
struct CgLauf {
  size_t iterationen = 0;
  bool nicht_konvergiert = false;
  double rest = 0;
};
CgLauf cpu_loese(const System& sys, const std::vector<std::optional<Fest>>& fest, std::vector<V3>& dv);
M3 m3_inv(const M3& m);
V3 m3_mal(const M3& m, V3 v);

// sim/src/implizit.rs:457-531
struct ImplizitParameter {
  size_t schritte_je_bild = 5;
  size_t cg_max = 50;
  double cg_toleranz = 1e-5;
  double naht_k = 500.0;
  double kontakt_rand = 1e-4;
  bool normalkraft_aus_last = false;
  bool durchstoss_pruefen = true;
  bool selbstkollision = false;  // proximity stage only (selbstkollision.rs:387-788)
  double selbst_zusatzdicke = 2.5e-3;
  double selbst_steifigkeit = 1e-3;
  size_t selbst_stoss_iterationen = 1;      // implizit.rs:491, 525
  bool selbst_schnitte_an_naehten = false;  // implizit.rs:494, 526
  size_t koerperpunkt_durchgaenge = 0;      // implizit.rs:479, 520
  double koerperpunkt_tiefe = 0.01;         // implizit.rs:481, 521
};
// sim/src/implizit.rs:535-561
struct ImplizitStatistik {
  size_t selbst_stoesse = 0, durchdringungen = 0, durchdringungsgebiete = 0;
  size_t cg_iterationen = 0, loesungen = 0, nicht_konvergiert = 0, kontakte = 0, haftend = 0,
         freigegeben = 0, durchstoesse = 0, koerperpunkte = 0, naehe_punkt_dreieck = 0, naehe_kante_kante = 0;
  double rest_max = 0;
};
// Forward record of one substep, for the adjoint (no reference counterpart):
// the state at the start, the final solution, the contact set of the last
// solve and after the release pass, each held point's normal force and
// friction case, and per point which bodies pushed it out after the move.
struct Aufnahme {
  double h = 0;
  std::vector<V3> x, v, dv;
  std::vector<std::optional<Fest>> fest;       // after the release pass (friction)
  std::vector<std::optional<Fest>> fest_loes;  // in the last solve (a second release pass ends the loop)
  std::vector<double> fn;
  std::vector<uint8_t> reib;    // held points: 1 stick, 2 slip
  std::vector<uint32_t> stoss;  // body b: bit 2b pushed out, bit 2b+1 inward normal velocity removed
  std::vector<Koerper> koerper; // the bodies as placed for this substep
};
// Parameter cotangents per element, summed over the substeps of a backward
// pass: membranes (E_warp, E_weft, G, rotation of the grain basis), hinges k.
struct AdjGrad {
  std::vector<std::array<double, 4>> membran;
  std::vector<double> biegung;
};
struct AdjStat {
  size_t cg_iterationen = 0, loesungen = 0, nicht_konvergiert = 0;
};

// sim/src/implizit.rs:570-1057
struct ImplizitCg {
  ImplizitParameter param;
  ImplizitStatistik statistik;
  std::vector<V3> dv_vorher;
  std::optional<std::pair<Stoffnetz, Stoffwerte>> selbst;
  std::vector<uint32_t> folge;     // per triangle: steps in a row with an edge through it
  std::vector<Schnitt> schnitte;   // of the last system build
  System system_bauen(Szene& s, double h, std::vector<std::optional<Fest>>& fest);
  void schritt(Szene& s, double h, Aufnahme* auf = nullptr);
  void bild(Szene& s, std::vector<Aufnahme>* auf = nullptr);
  std::vector<V3> op(Szene& s, const std::vector<V3>& p);
  // Adjoint of one recorded substep (adjoint.cpp): xq, vq enter as the
  // cotangents of the substep's output x, v and leave as those of its input;
  // lam is the adjoint solve's warm start and result.
  void adjoint_schritt(Szene& s, const Aufnahme& a, std::vector<V3>& xq, std::vector<V3>& vq, AdjGrad& g,
                       std::vector<V3>& lam, AdjStat& st, double adj_toleranz);
};

// ---------------------------------------------------------------- measurement
// sim/src/messung.rs:10-116
double umfang_in_ebene(const Szene& s, V3 punkt, V3 normale);
std::vector<std::pair<double, double>> dehnung_je_dreieck(const Szene& s);
double nahtspalt(const Szene& s);
double mittlere_geschwindigkeit(const Szene& s);
V3 schwerpunkt(const Szene& s);

// ---------------------------------------------------------------- XPBD cross-check
// sim/src/cpu.rs:62-245 (CpuReferenz); the device step has no XPBD form
struct Kontaktstatistik {
  size_t kontakte = 0, haftend = 0;
  double tiefe = 0, tangential = 0;
};
void xpbd_abstand(const std::vector<V3>& x, const std::vector<V3>& delta, std::vector<V3>& korr,
                  const std::vector<double>& w, std::array<uint32_t, 2> p, double ruhe, double alpha_h2);
void xpbd_biegung(const std::vector<V3>& x, const std::vector<V3>& delta, std::vector<V3>& korr,
                  const std::vector<double>& w, std::array<uint32_t, 4> p, double ruhe, double alpha_h2);
struct CpuReferenz {
  std::vector<V3> delta, korr, last;
  Kontaktstatistik statistik;
  void unterschritt(Szene& s, double h);
  void bild(Szene& s, size_t unterschritte);
};

}  // namespace orc
