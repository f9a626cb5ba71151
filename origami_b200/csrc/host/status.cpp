#include "status.h"

namespace {
thread_local std::string t_last_error;
}

og_status og_fail(og_status st, const std::string& msg) {
  t_last_error = msg;
  return st;
}

extern "C" {

const char* og_last_error(void) { return t_last_error.c_str(); }

const char* og_status_string(int s) {
  switch (s) {
    case OG_OK: return "ok";
    case OG_E_BADARG: return "bad argument";
    case OG_E_NONFINITE: return "non-finite velocity or force (diverged)";
    case OG_E_SHAKE: return "SHAKE did not converge";
    case OG_E_TIMEOUT: return "bounded device wait timed out";
    case OG_E_CUDA: return "CUDA error";
    case OG_E_NOMEM: return "out of memory";
    case OG_E_STATE: return "invalid engine state";
    case OG_E_DATA: return "force-field or template data error";
    case OG_E_UNSUPPORTED: return "unsupported";
    case OG_E_IO: return "file i/o error";
    default: return "unknown status";
  }
}

const char* og_version(void) { return "origami-b200 0.1 (sm_100a)"; }

}  // extern "C"
