// Adjoint schedules (the transpose / conjugate transpose of a plan's linear
// map, same scale), used for differentiation.
//
//   plan kind   adjoint                                  weights
//   C2C dir     C2C -dir                                 -
//   R2C         C2R                                      input bins 0<k<n/2 halved
//   C2R         R2C                                      output bins 0<k<n/2 doubled
//   DCT-I       DCT-I                                    inner elements /2 in, *2 out
//   DCT-II      DCT-III                                  input element 0 doubled
//   DCT-III     DCT-II                                   output element 0 halved
//   DST-II      DST-III                                  input element n-1 doubled
//   DST-III     DST-II                                   output element n-1 halved
//   DCT-IV, DST-I, DST-IV, DHT: symmetric matrices, self-adjoint
//   R2HC        HC2R                                     half-complex inputs (not 0, n/2) halved
//   HC2R        R2HC                                     half-complex outputs (not 0, n/2) doubled
// Rader and Bluestein plans need nothing special: the adjoint of a C2C of
// any length is the opposite-direction C2C of that length.
#include "plan.hpp"

namespace plfft_b200 {

std::unique_ptr<Node> make_adjoint_node(const ConfigData& c, std::string* why) {
  // the adjoint reads the plan's output layout and writes its input layout
  const Layout lay{c.howmany, c.ostride, c.howmany > 1 ? c.odist : 0, c.istride, c.howmany > 1 ? c.idist : 0};
  const float scale = float(c.scale);
  if (c.data_type != PLFFT_DATA_TYPE_FP32) {
    if (why) *why = "adjoint available for FP32 plans";
    return nullptr;
  }
  switch (c.kind) {
    case TKind::C2C:
      return make_c2c_node(c.n, lay, -c.payload, scale, c.precision, why);
    case TKind::R2C:  // one fused kernel where it applies
      if (auto f = make_real_fused_node(FR_C2R, c.n, lay, scale, 1)) return f;
      return make_realwrap_node(RW_C2R, c.n, lay, scale, why, AW_HERM_HALF, AW_NONE);
    case TKind::C2R:
      if (auto f = make_real_fused_node(FR_R2C, c.n, lay, scale, 2)) return f;
      return make_realwrap_node(RW_R2C, c.n, lay, scale, why, AW_NONE, AW_HERM_DOUBLE);
    case TKind::R2R:
      switch (c.payload) {
        case PLFFT_R2R_DCT_1: return make_realwrap_node(RW_DCT1, c.n, lay, scale, why, AW_INNER_HALF, AW_INNER_X2);
        case PLFFT_R2R_DCT_2:
          if (auto f = make_real_fused_node(FR_DCT3, c.n, lay, scale, 3)) return f;
          return make_realwrap_node(RW_DCT3, c.n, lay, scale, why, AW_FIRST_X2, AW_NONE);
        case PLFFT_R2R_DCT_3: return make_realwrap_node(RW_DCT2, c.n, lay, scale, why, AW_NONE, AW_FIRST_HALF);
        case PLFFT_R2R_DCT_4:  // self-adjoint
          if (auto f = make_real_fused_node(FR_DCT4, c.n, lay, scale)) return f;
          return make_realwrap_node(RW_DCT4, c.n, lay, scale, why);
        case PLFFT_R2R_DST_1: return make_realwrap_node(RW_DST1, c.n, lay, scale, why);
        case PLFFT_R2R_DST_2:
          if (auto f = make_real_fused_node(FR_DST3, c.n, lay, scale, 3)) return f;
          return make_realwrap_node(RW_DST3, c.n, lay, scale, why, AW_LAST_X2, AW_NONE);
        case PLFFT_R2R_DST_3: return make_realwrap_node(RW_DST2, c.n, lay, scale, why, AW_NONE, AW_LAST_HALF);
        case PLFFT_R2R_DST_4:
          if (auto f = make_real_fused_node(FR_DST4, c.n, lay, scale)) return f;
          return make_realwrap_node(RW_DST4, c.n, lay, scale, why);
        case PLFFT_R2R_DHT:  // self-adjoint
          if (auto f = make_real_fused_node(FR_DHT, c.n, lay, scale)) return f;
          return make_realwrap_node(RW_DHT, c.n, lay, scale, why);
        case PLFFT_R2R_R2HC: return make_realwrap_node(RW_HC2R, c.n, lay, scale, why, AW_HC_HALF, AW_NONE);
        case PLFFT_R2R_HC2R: return make_realwrap_node(RW_R2HC, c.n, lay, scale, why, AW_NONE, AW_HC_DOUBLE);
      }
      break;
  }
  if (why) *why = "no adjoint for this transform";
  return nullptr;
}

}  // namespace plfft_b200
