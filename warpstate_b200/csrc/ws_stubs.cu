#include "ws_internal.h"
extern "C" {
ws_status ws_scan_batch(ws_matcher*, const ws_item*, uint64_t, ws_tagged_match*, uint64_t, uint64_t*, ws_error_info*) { return WS_ERR_DEVICE; }
ws_status ws_stream_begin(ws_matcher*, ws_stream**, ws_error_info*) { return WS_ERR_DEVICE; }
ws_status ws_stream_feed(ws_stream*, const uint8_t*, uint64_t, ws_match64*, uint64_t, uint64_t*, ws_error_info*) { return WS_ERR_DEVICE; }
ws_status ws_stream_end(ws_stream*, ws_match64*, uint64_t, uint64_t*, ws_error_info*) { return WS_ERR_DEVICE; }
void ws_stream_destroy(ws_stream*) {}
}
