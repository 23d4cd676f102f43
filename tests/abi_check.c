/* Compiled by tests/test_abi.py as plain C99 against include/lvbh.h and linked with liblvbh.so:
 * proves the header is C, prints the struct layout the ctypes binding must match, and calls
 * the entry points that need no GPU. */
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include "lvbh.h"

int main(void) {
    lvbh_result r;
    memset(&r, 0, sizeof r);
    printf("sizeof_result %zu\n", sizeof(lvbh_result));
    printf("off_nodes %zu\n", offsetof(lvbh_result, nodes));
    printf("off_bounds %zu\n", offsetof(lvbh_result, bounds));
    printf("off_owned %zu\n", offsetof(lvbh_result, owned));
    printf("sizeof_config %zu\n", sizeof(lvbh_config));
    printf("version %s\n", lvbh_version());
    printf("build_null_ctx %d\n", lvbh_build_soup(NULL, NULL, 0, NULL, 0, &r, NULL));
    printf("indexed_null_ctx %d\n", lvbh_build_indexed(NULL, NULL, 0, NULL, 0, NULL, 0, &r, NULL));
    printf("sync_null %d\n", lvbh_sync(NULL));
    printf("release_null %d\n", lvbh_release(NULL, NULL));
    printf("create_null %d\n", lvbh_create(NULL, NULL));
    printf("stage_null %d\n", lvbh_stage_times(NULL, NULL));
    printf("trace_null %d\n", lvbh_trace(NULL, NULL, NULL, 0, NULL, 0, NULL, NULL, NULL, NULL));
    printf("copy_null %d\n", lvbh_copy_to_host(NULL, NULL, NULL, 0, NULL));
    printf("last_error_null %s\n", lvbh_last_error(NULL));
    printf("scratch_1M %zu\n", lvbh_scratch_bytes(1u << 20));
    printf("batched_null_ctx %d\n", lvbh_build_batched(NULL, NULL, NULL, 0, NULL, NULL, 0, &r, NULL));
    printf("sizeof_server_config %zu\n", sizeof(lvbh_server_config));
    printf("sizeof_tunables %zu\n", sizeof(lvbh_tunables));
    printf("set_tunables_null %d\n", lvbh_set_tunables(NULL, NULL));
    printf("get_tunables_null %d\n", lvbh_get_tunables(NULL, NULL, NULL, NULL));
    printf("sizeof_request_info %zu\n", sizeof(lvbh_request_info));
    printf("off_latency %zu\n", offsetof(lvbh_request_info, latency_ms));
    printf("sizeof_server_stats %zu\n", sizeof(lvbh_server_stats));
    printf("off_max_batch_seen %zu\n", offsetof(lvbh_server_stats, max_batch_seen));
    {
        const float *tri = NULL;
        uint32_t n = 0;
        double b6[6];
        uint64_t line = 7;
        lvbh_pt_frame fr;
        memset(&fr, 0, sizeof fr);
        printf("sizeof_pt_frame %zu\n", sizeof(lvbh_pt_frame));
        printf("mesh_null_ctx %d\n", lvbh_build_mesh(NULL, NULL, 0, NULL, 0, NULL, 0, &r, NULL));
        printf("trace_mesh_null_ctx %d\n", lvbh_trace_mesh(NULL, NULL, NULL, NULL, 0, 0, NULL, 0, NULL, NULL, NULL, NULL));
        printf("pt_null_ctx %d\n", lvbh_pt_sample(NULL, NULL, NULL, 0, NULL, NULL, 1, 1, &fr, NULL));
        printf("parse_obj_null_ctx %d\n", lvbh_parse_obj(NULL, "v 0 0 0\n", 8, LVBH_INPUT_HOST, &tri, &n, b6, &line, NULL));
    }
    {
        uint64_t t = 0;
        printf("server_create_null %d\n", lvbh_server_create(NULL, NULL));
        printf("submit_null %d\n", lvbh_submit(NULL, NULL, 0, NULL, 0, &t));
        printf("poll_null %d\n", lvbh_poll(NULL, 1, NULL, NULL));
        printf("wait_null %d\n", lvbh_wait(NULL, 1, 0, NULL, NULL));
        printf("release_req_null %d\n", lvbh_request_release(NULL, 1));
        printf("stats_null %d\n", lvbh_server_stats_get(NULL, NULL));
        printf("server_error_null %s\n", lvbh_server_last_error(NULL));
        lvbh_server_destroy(NULL);
    }
    return 0;
}
