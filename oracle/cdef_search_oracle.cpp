// cdef_search_oracle.cpp - CPU oracle for goav1's encoder CDEF strength search
// (internal/av1/encoder/cdef_search.go).  Test infrastructure only.
#include "pf_oracle.h"

extern "C" int oracle_cdef_search(const pf_frame*, const pf_frame*, const uint8_t*, const pf_cdef_search_params*,
                                  uint64_t*, uint8_t*, pf_cdef_search_result*) {
  return PF_ERR_UNSUPPORTED;
}

extern "C" int oracle_cdef_unit_sse(const pf_frame*, const pf_frame*, const uint8_t*, int, int, int, int, int,
                                    uint64_t*) {
  return PF_ERR_UNSUPPORTED;
}
