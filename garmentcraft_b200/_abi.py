"""ctypes mirrors of the C ABI structs in include/klon3d_step.h.

Field order and types follow the header exactly; a CPU test checks the sizes
against the compiled library.
"""
import ctypes as C

c_f64_p = C.POINTER(C.c_double)
c_u32_p = C.POINTER(C.c_uint32)
c_u8_p = C.POINTER(C.c_uint8)
c_f32_p = C.POINTER(C.c_float)

K3D_ABI_VERSION = 4

K3D_OK = 0
K3D_NOT_CONVERGED = 1
K3D_BREAKDOWN = 2
K3D_NON_FINITE = 3
K3D_DEVICE_ERROR = 4
K3D_BAD_ARGUMENT = 5
K3D_TIMEOUT = 6

K3D_FP64 = 0
K3D_MIXED = 1
K3D_MIXED_STORAGE = 2

K3D_BODY_CYLINDER = 0
K3D_BODY_SDF_GRID = 1
K3D_BODY_MESH = 2

STATUS_NAMES = {
    0: "K3D_OK", 1: "K3D_NOT_CONVERGED", 2: "K3D_BREAKDOWN", 3: "K3D_NON_FINITE",
    4: "K3D_DEVICE_ERROR", 5: "K3D_BAD_ARGUMENT", 6: "K3D_TIMEOUT",
}


class K3dParams(C.Structure):
    _fields_ = [
        ("schritte_je_bild", C.c_int32),
        ("cg_max", C.c_int32),
        ("cg_toleranz", C.c_double),
        ("naht_k", C.c_double),
        ("kontakt_rand", C.c_double),
        ("normalkraft_aus_last", C.c_int32),
        ("durchstoss_pruefen", C.c_int32),
        ("selbstkollision", C.c_int32),
        ("precision", C.c_int32),
        ("selbst_zusatzdicke", C.c_double),
        ("selbst_steifigkeit", C.c_double),
        ("selbst_stoss_iterationen", C.c_int32),
        ("selbst_schnitte_an_naehten", C.c_int32),
        ("koerperpunkt_durchgaenge", C.c_int32),
        ("pcg_bloecke", C.c_int32),
        ("koerperpunkt_tiefe", C.c_double),
        ("graph", C.c_int32),
        ("pcg_threads", C.c_int32),
    ]


class K3dSimparams(C.Structure):
    _fields_ = [
        ("bild_dt", C.c_double),
        ("schwerkraft", C.c_double * 3),
        ("daempfung", C.c_double),
    ]


class K3dBody(C.Structure):
    _fields_ = [
        ("art", C.c_int32),
        ("dims", C.c_int32 * 3),
        ("punkt", C.c_double * 3),
        ("achse", C.c_double * 3),
        ("radius", C.c_double),
        ("geschwindigkeit", C.c_double * 3),
        ("ursprung", C.c_double * 3),
        ("spacing", C.c_double),
        ("sdf", c_f32_p),
        ("instanz", C.c_int32),
        ("pad", C.c_int32),
        ("netz", C.c_void_p),
    ]


class K3dScene(C.Structure):
    _fields_ = [
        ("n_punkte", C.c_int64),
        ("x", c_f64_p),
        ("v", c_f64_p),
        ("masse", c_f64_p),
        ("w", c_f64_p),
        ("kollisionsabstand", c_f64_p),
        ("reibung", c_f64_p),
        ("n_abstand", C.c_int64),
        ("abstand_punkte", c_u32_p),
        ("abstand_ruhe", c_f64_p),
        ("abstand_nachgiebigkeit", c_f64_p),
        ("membran_kante", c_u8_p),
        ("n_naht", C.c_int64),
        ("naht_punkte", c_u32_p),
        ("naht_ruhe", c_f64_p),
        ("n_biegung", C.c_int64),
        ("biegung_punkte", c_u32_p),
        ("biegung_ruhe", c_f64_p),
        ("biegung_nachgiebigkeit", c_f64_p),
        ("n_membran", C.c_int64),
        ("membran_punkte", c_u32_p),
        ("membran_flaeche", c_f64_p),
        ("membran_ruhe_inv", c_f64_p),
        ("membran_kette", c_f64_p),
        ("membran_schuss", c_f64_p),
        ("membran_steif", c_f64_p),
        ("n_dreiecke", C.c_int64),
        ("dreiecke", c_u32_p),
        ("ruhe_inv", c_f64_p),
        ("n_koerper", C.c_int32),
        ("pad0", C.c_int32),
        ("koerper", C.POINTER(K3dBody)),
        ("param", K3dSimparams),
        ("zeit", C.c_double),
        ("n_teile", C.c_int64),
        ("teil_bereiche", C.POINTER(C.c_int64)),
        ("teil_dehnung", c_f64_p),
        ("teil_band_von", C.POINTER(C.c_int32)),
        ("n_instanzen", C.c_int64),
        ("instanz_punkte", C.POINTER(C.c_int64)),
    ]


class K3dStats(C.Structure):
    _fields_ = [
        ("cg_iterationen", C.c_int64),
        ("loesungen", C.c_int64),
        ("nicht_konvergiert", C.c_int64),
        ("kontakte", C.c_int64),
        ("haftend", C.c_int64),
        ("freigegeben", C.c_int64),
        ("durchstoesse", C.c_int64),
        ("koerperpunkte", C.c_int64),
        ("rest_max", C.c_double),
        ("naehe_punkt_dreieck", C.c_int64),
        ("naehe_kante_kante", C.c_int64),
        ("selbst_stoesse", C.c_int64),
        ("durchdringungen", C.c_int64),
        ("durchdringungsgebiete", C.c_int64),
        ("zusammenbrueche", C.c_int64),
        ("dv_max", C.c_double),
    ]


class K3dAdjointStats(C.Structure):
    _fields_ = [
        ("cg_iterationen", C.c_int64),
        ("loesungen", C.c_int64),
        ("nicht_konvergiert", C.c_int64),
        ("zusammenbrueche", C.c_int64),
        ("ms_vorwaerts", C.c_double),
        ("ms_rueckwaerts", C.c_double),
        ("ms_neuberechnung", C.c_double),
    ]


class K3dMeshInfo(C.Structure):
    _fields_ = [
        ("n_punkte", C.c_int64),
        ("n_dreiecke", C.c_int64),
        ("randkanten", C.c_int64),
        ("volumen", C.c_double),
        ("suchtiefe", C.c_double),
        ("gitter_ursprung", C.c_double * 3),
        ("gitter_zelle", C.c_double),
        ("gitter_zahl", C.c_int64 * 3),
        ("gitter_eintraege", C.c_int64),
        ("ms_letzter_aufruf", C.c_double),
        ("kernels_letzter_aufruf", C.c_int64),
        ("ungeklaert", C.c_int64),
    ]


class K3dContactSet(C.Structure):
    _fields_ = [
        ("fest", C.POINTER(C.c_uint8)),
        ("normale", C.POINTER(C.c_double)),
        ("vn_soll", C.POINTER(C.c_double)),
    ]


class K3dCgResult(C.Structure):
    _fields_ = [
        ("iterationen", C.c_int64),
        ("nicht_konvergiert", C.c_int32),
        ("breakdown", C.c_int32),
        ("rest", C.c_double),
    ]


class K3dSystemReadback(C.Structure):
    _fields_ = [
        ("rhs", c_f64_p),
        ("f", c_f64_p),
        ("last", c_f64_p),
        ("pinv", c_f64_p),
        ("normale", c_f64_p),
        ("vn_soll", c_f64_p),
        ("fest", c_u8_p),
    ]


class K3dMaterial(C.Structure):
    _fields_ = [
        ("dehnung_n_m", C.c_double),
        ("kette_n_m", C.c_double),
        ("schub_n_m", C.c_double),
        ("biegung_nm", C.c_double),
        ("biegung_kette_nm", C.c_double),
        ("biegung_schraege_nm", C.c_double),
        ("flaechengewicht_kg_m2", C.c_double),
        ("dicke_m", C.c_double),
        ("reibung", C.c_double),
    ]


class K3dPiece(C.Structure):
    _fields_ = [
        ("n_punkte", C.c_int64),
        ("punkte_mm", c_f64_p),
        ("n_dreiecke", C.c_int64),
        ("dreiecke", c_u32_p),
        ("fadenlauf", C.c_double * 2),
        ("material", K3dMaterial),
        ("reduktion", C.c_double),
        ("lage", c_f64_p),
    ]


class K3dSeamPart(C.Structure):
    _fields_ = [
        ("teil_a", C.c_int32),
        ("teil_b", C.c_int32),
        ("n_paare", C.c_int64),
        ("paare", c_u32_p),
    ]


class K3dSeam(C.Structure):
    _fields_ = [
        ("n_teilnaehte", C.c_int32),
        ("pad0", C.c_int32),
        ("teilnaehte", C.POINTER(K3dSeamPart)),
        ("laenge_a_mm", C.c_double),
        ("laenge_b_mm", C.c_double),
    ]


class K3dPattern(C.Structure):
    _fields_ = [
        ("n_teile", C.c_int32),
        ("n_naehte", C.c_int32),
        ("teile", C.POINTER(K3dPiece)),
        ("naehte", C.POINTER(K3dSeam)),
        ("param", K3dSimparams),
        ("naht_nachgiebigkeit", C.c_double),
        ("einhalteweite", C.c_int32),
        ("pad0", C.c_int32),
    ]


def ptr(a, ctype):
    """Pointer to a contiguous numpy array (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))
