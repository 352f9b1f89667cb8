"""Host logic of the launch-shape tuner: candidates, cache key, cache file."""
from garmentcraft_b200 import autotune
from garmentcraft_b200.params import ImplizitParameter
from garmentcraft_b200 import synth
from garmentcraft_b200.implizit import build_scene
from garmentcraft_b200.szene import Szene


def test_kandidaten():
    assert autotune.kandidaten(148) == [148, 74, 37, 18, 9]
    assert autotune.kandidaten(296, instanzen=20) == [296, 148, 74, 37]
    assert autotune.kandidaten(6) == [6]


def test_schluessel_und_instanzen():
    m, k = synth.sheet_over_sphere(n=9, seed=1)
    s = build_scene(m, [k])
    p = ImplizitParameter()
    a = autotune.schluessel("B200 (f64)", p, s)
    assert a == f"B200 (f64)|p0|n{s.n}|t{len(s.dreiecke)}|i1|s5|sk0"
    b = Szene.verbinden([s.copy(), s.copy()])
    assert autotune._instanzen(b) == 2
    assert autotune.schluessel("B200 (f64)", p, b) != a


def test_cache_rundreise(tmp_path, monkeypatch):
    pfad = str(tmp_path / "sub" / "t.json")
    monkeypatch.setenv(autotune.CACHE_ENV, pfad)
    assert autotune.cache_pfad() == pfad
    assert autotune._lesen(pfad) == {}
    autotune._schreiben(pfad, {"k": {"pcg_bloecke": 37, "graph": True}})
    assert autotune._lesen(pfad) == {"k": {"pcg_bloecke": 37, "graph": True}}
