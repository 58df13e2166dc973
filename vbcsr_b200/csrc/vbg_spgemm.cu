// Entry points whose device implementation lives in later translation units.
#include "vbg_internal.cuh"
using namespace vbg;
extern "C" {
int vbg_matrix_axpby(vbg_matrix*, double, double, const vbg_matrix*, double, double, void*) {
  return fail(VBG_E_STATE, "vbg_matrix_axpby: not built yet");
}
int vbg_matrix_filter_blocks(vbg_matrix*, double, void*) { return fail(VBG_E_STATE, "not built yet"); }
int vbg_matrix_transpose(const vbg_matrix*, vbg_matrix**, void*) { return fail(VBG_E_STATE, "not built yet"); }
int vbg_spgemm(const vbg_matrix*, const vbg_matrix*, double, vbg_matrix**, int64_t*, void*) {
  return fail(VBG_E_STATE, "not built yet");
}
}
