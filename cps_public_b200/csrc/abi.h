// abi.h -- helpers shared by the translation units that implement the C ABI
// (capi.cu, serve.cu): the gauge handle, error capture and argument checks.
#pragma once
#include <string>

#include "host.h"

struct cpsb_gauge_s {
  cpsb::Gauge g;
};

namespace cpsb {

// Message of the last failed call on this thread (cpsb_last_error).
std::string &last_error_slot();

// Runs f, converting library errors into status codes.
template <class F>
int guarded(F &&f) {
  try {
    return f();
  } catch (const Error &e) {
    last_error_slot() = e.msg;
    return e.code;
  } catch (const std::bad_alloc &) {
    last_error_slot() = "host allocation failed";
    return CPSB_ERR_OOM;
  } catch (...) {
    last_error_slot() = "unexpected exception";
    return CPSB_ERR_CUDA;
  }
}

void need_init();
void check_params(cpsb_gauge h, const cpsb_dirac_params *p);
void check_cg(const cpsb_cg_arg *a);
// Sites of one checkerboard vector (4-D half volume x Ls).
long cb_sites(cpsb_gauge h, const cpsb_dirac_params *p);
// Geometry (column layout) of the checkerboard fields of this operator.
Geom geom_of(cpsb_gauge h, const cpsb_dirac_params *p, int nrhs);

}  // namespace cpsb
