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
    return 0;
}
