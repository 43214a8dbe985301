// rc_server.cu -- continuous-batching solve server (placeholder until the
// scheduler lands; every entry point reports RC_E_STATE).
#include "radchan.h"

extern "C" {
int rc_server_create(int, double, int, rc_server **out) {
    if (out) *out = nullptr;
    return RC_E_STATE;
}
int rc_server_add_tables(rc_server *, const rc_tables *, int *) { return RC_E_STATE; }
int rc_server_submit(rc_server *, const rc_request *, int64_t *) { return RC_E_STATE; }
int rc_server_wait(rc_server *, int64_t, float *, float *, rc_result_info *) { return RC_E_STATE; }
int rc_server_stats(rc_server *, double *, double *, double *) { return RC_E_STATE; }
int rc_server_destroy(rc_server *) { return RC_OK; }
}
