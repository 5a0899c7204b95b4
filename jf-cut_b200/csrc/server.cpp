// server.cpp — placeholder until the continuous-batching server lands.
#include "engine.h"

struct jfc_server { jfc_ctx* ctx; };

extern "C" {
int jfc_server_create(jfc_ctx* ctx, size_t, int, jfc_server** out) {
  if (!ctx || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  *out = new jfc_server{ctx};
  return JFC_OK;
}
void jfc_server_destroy(jfc_server* s) { delete s; }
int jfc_server_submit(jfc_server*, int, int, int, int, const void*, int, const uint8_t*, const jfc_model*, int*) {
  return set_error(JFC_ERR_STATE, "server not available");
}
int jfc_server_edit(jfc_server*, int, const uint32_t*, const uint8_t*, size_t) {
  return set_error(JFC_ERR_STATE, "server not available");
}
int jfc_server_wait(jfc_server*, int, int, jfc_request_info*) { return set_error(JFC_ERR_STATE, "server not available"); }
int jfc_server_read_labels(jfc_server*, int, uint8_t*) { return set_error(JFC_ERR_STATE, "server not available"); }
int jfc_server_close(jfc_server*, int) { return set_error(JFC_ERR_STATE, "server not available"); }
int jfc_server_cancel(jfc_server*, int) { return set_error(JFC_ERR_STATE, "server not available"); }
}
