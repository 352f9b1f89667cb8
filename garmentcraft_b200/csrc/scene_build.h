// Host-side scene built from a pattern (internal).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/klon3d_step.h"

namespace k3d {

struct BuiltScene {
  std::vector<double> x, v, masse, w, kabst, reib;
  std::vector<uint32_t> a_p, n_p, b_p, m_punkte, dreiecke;
  std::vector<double> a_r, a_a, n_r, b_r, b_a;
  std::vector<uint8_t> mkante;
  std::vector<double> m_flaeche, m_ruhe_inv, m_kette, m_schuss, m_steif, ruhe_inv;
  std::vector<int64_t> teil_bereiche;  // 4 per piece
  std::vector<double> teil_dehnung;
  std::vector<int32_t> teil_band_von;
  k3d_simparams param{};
  size_t membran_entartet = 0, naht_biegung_ohne = 0, einhalte_kanten = 0;
  size_t farben[3] = {0, 0, 0};
};

k3d_status build_scene_impl(const k3d_pattern* pat, BuiltScene& out);
void built_scene_view(BuiltScene& s, k3d_scene* out);

}  // namespace k3d

struct k3d_built_scene {
  k3d::BuiltScene s;
};
