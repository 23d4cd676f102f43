// lvbh_napi.cc - Node.js N-API binding of the LBVH builder's C ABI (include/lvbh.h).
//
// UNVERIFIED: this environment has neither a `node` binary nor node_api.h, so this file is
// not compiled or run by the build or the tests; the C ABI it wraps is tested from C
// (tests/abi_check.c) and Python (ctypes).  Build with node-gyp (binding.gyp beside it).
//
// It mirrors the reference's JavaScript entry (scripts/bvh/build-bvh.js:1-66):
//
//   const { initBVHBuild } = require('./lvbh_napi.node')
//   const BVH = initBVHBuild(0)                            // CUDA device ordinal
//   const { BVH_BUFFER, O_TRIANGLE_BUFFER } = await BVH.build(TRI_ARRAY, NUM_TRIS, BOUNDS)
//   const { NUM_TRIS, TRI_ARR, BOUNDS } = await BVH.parseObj(fileText)   // parse-obj.js:3-88
//
// TRI_ARRAY is a JS number array or a Float32Array (12 floats per triangle); BOUNDS is
// {min: [x, y, z], max: [x, y, z]} (parse-obj.js:80-87) or undefined (device reduction).
// The results come back as ArrayBuffers in the reference's layouts (64-byte BVHNode records,
// 48-byte triangles), ready for device.queue.writeBuffer into the path tracer's storage
// buffers: a WebGPU buffer cannot alias CUDA memory, so the node and triangle buffers cross
// the host once.  As in the reference, a TRI_ARRAY longer than 12 * NUM_TRIS throws a
// RangeError (Float32Array.set, build-bvh.js:20).
#include <node_api.h>

#include <cstring>
#include <string>
#include <vector>

#include "lvbh.h"

namespace {

#define NAPI_OK(env, call)                                              \
    do {                                                                \
        if ((call) != napi_ok) {                                        \
            napi_throw_error((env), nullptr, "N-API call failed: " #call); \
            return nullptr;                                             \
        }                                                               \
    } while (0)

struct Builder {
    lvbh_ctx *ctx = nullptr;
};

struct Job {
    Builder *b = nullptr;
    std::vector<float> tri;
    uint32_t n = 0;
    bool has_bounds = false;
    float bounds[6] = {};
    std::vector<char> nodes, tris;
    int status = LVBH_OK;
    std::string error;
    napi_deferred deferred = nullptr;
    napi_async_work work = nullptr;
};

void finalize_builder(napi_env, void *data, void *) {
    auto *b = static_cast<Builder *>(data);
    lvbh_destroy(b->ctx);
    delete b;
}

// Worker thread: build on the GPU, copy the two buffers the path tracer consumes to the host.
void execute(napi_env, void *data) {
    auto *j = static_cast<Job *>(data);
    lvbh_result r;
    std::memset(&r, 0, sizeof r);
    j->status = lvbh_build_soup(j->b->ctx, j->tri.data(), j->n, j->has_bounds ? j->bounds : nullptr,
                                LVBH_INPUT_HOST, &r, nullptr);
    if (j->status != LVBH_OK) {
        j->error = lvbh_last_error(j->b->ctx);
        return;
    }
    j->nodes.resize(64ull * j->n);
    j->tris.resize(48ull * j->n);
    if (j->n && (lvbh_copy_to_host(j->b->ctx, j->nodes.data(), r.nodes, j->nodes.size(), nullptr) ||
                 lvbh_copy_to_host(j->b->ctx, j->tris.data(), r.tris, j->tris.size(), nullptr))) {
        j->status = LVBH_ECUDA;
        j->error = lvbh_last_error(j->b->ctx);
    }
    lvbh_release(j->b->ctx, &r);
}

void complete(napi_env env, napi_status, void *data) {
    auto *j = static_cast<Job *>(data);
    if (j->status != LVBH_OK) {
        napi_value msg, err;
        napi_create_string_utf8(env, j->error.c_str(), NAPI_AUTO_LENGTH, &msg);
        napi_create_error(env, nullptr, msg, &err);
        napi_reject_deferred(env, j->deferred, err);
    } else {
        napi_value out, nodes, tris;
        void *p = nullptr;
        napi_create_object(env, &out);
        napi_create_arraybuffer(env, j->nodes.size(), &p, &nodes);
        if (!j->nodes.empty()) std::memcpy(p, j->nodes.data(), j->nodes.size());
        napi_create_arraybuffer(env, j->tris.size(), &p, &tris);
        if (!j->tris.empty()) std::memcpy(p, j->tris.data(), j->tris.size());
        napi_set_named_property(env, out, "BVH_BUFFER", nodes);
        napi_set_named_property(env, out, "O_TRIANGLE_BUFFER", tris);
        napi_resolve_deferred(env, j->deferred, out);
    }
    napi_delete_async_work(env, j->work);
    delete j;
}

// build(TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS) -> Promise<{BVH_BUFFER, O_TRIANGLE_BUFFER}>
napi_value build(napi_env env, napi_callback_info info) {
    size_t argc = 3;
    napi_value argv[3], self;
    void *data = nullptr;
    NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, &self, &data));
    auto *b = static_cast<Builder *>(data);
    auto *j = new Job();
    j->b = b;
    double nd = 0;
    NAPI_OK(env, napi_get_value_double(env, argv[1], &nd));
    j->n = static_cast<uint32_t>(nd);
    j->tri.assign(12ull * j->n, 0.0f);
    bool is_typed = false;
    napi_is_typedarray(env, argv[0], &is_typed);
    if (is_typed) {
        napi_typedarray_type type;
        size_t len = 0;
        void *raw = nullptr;
        NAPI_OK(env, napi_get_typedarray_info(env, argv[0], &type, &len, &raw, nullptr, nullptr));
        if (len > j->tri.size()) {
            napi_throw_range_error(env, nullptr, "offset is out of bounds");
            delete j;
            return nullptr;
        }
        if (type == napi_float32_array) std::memcpy(j->tri.data(), raw, len * sizeof(float));
        else if (type == napi_float64_array)
            for (size_t i = 0; i < len; ++i) j->tri[i] = static_cast<float>(static_cast<double *>(raw)[i]);
    } else {
        uint32_t len = 0;
        NAPI_OK(env, napi_get_array_length(env, argv[0], &len));
        if (len > j->tri.size()) {
            napi_throw_range_error(env, nullptr, "offset is out of bounds");
            delete j;
            return nullptr;
        }
        for (uint32_t i = 0; i < len; ++i) {
            napi_value v;
            double x = 0;
            napi_get_element(env, argv[0], i, &v);
            napi_get_value_double(env, v, &x);
            j->tri[i] = static_cast<float>(x);  // Float32Array.set rounding
        }
    }
    napi_valuetype bt = napi_undefined;
    if (argc > 2) napi_typeof(env, argv[2], &bt);
    if (bt == napi_object) {
        const char *keys[2] = {"min", "max"};
        for (int h = 0; h < 2; ++h) {
            napi_value arr, v;
            NAPI_OK(env, napi_get_named_property(env, argv[2], keys[h], &arr));
            for (uint32_t a = 0; a < 3; ++a) {
                double x = 0;
                napi_get_element(env, arr, a, &v);
                napi_get_value_double(env, v, &x);
                j->bounds[3 * h + a] = static_cast<float>(x);  // DataView.setFloat32
            }
        }
        j->has_bounds = true;
    }
    napi_value promise, name;
    NAPI_OK(env, napi_create_promise(env, &j->deferred, &promise));
    napi_create_string_utf8(env, "lvbh.build", NAPI_AUTO_LENGTH, &name);
    NAPI_OK(env, napi_create_async_work(env, nullptr, name, execute, complete, j, &j->work));
    NAPI_OK(env, napi_queue_async_work(env, j->work));
    return promise;
}

// parseObj(text) on the GPU (scripts/obj/parse-obj.js:3-88): text is a string or a
// Uint8Array / ArrayBuffer of the file's UTF-8 bytes.  Resolves {NUM_TRIS, TRI_ARR (a
// Float32Array, 12 floats per triangle, floor included), BOUNDS: {min, max}}; rejects where the
// reference throws (LVBH_EPARSE; the message names the line).
struct ParseJob {
    Builder *b = nullptr;
    std::vector<char> text;
    std::vector<float> tri;
    uint32_t n = 0;
    double bounds[6] = {};
    int status = LVBH_OK;
    std::string error;
    napi_deferred deferred = nullptr;
    napi_async_work work = nullptr;
};

void parse_execute(napi_env, void *data) {
    auto *j = static_cast<ParseJob *>(data);
    const float *dtri = nullptr;
    uint64_t line = 0;
    j->status = lvbh_parse_obj(j->b->ctx, j->text.data(), j->text.size(), LVBH_INPUT_HOST, &dtri, &j->n,
                               j->bounds, &line, nullptr);
    if (j->status != LVBH_OK) {
        j->error = lvbh_last_error(j->b->ctx);
        return;
    }
    j->tri.resize(12ull * j->n);
    if (lvbh_copy_to_host(j->b->ctx, j->tri.data(), dtri, j->tri.size() * sizeof(float), nullptr)) {
        j->status = LVBH_ECUDA;
        j->error = lvbh_last_error(j->b->ctx);
    }
}

void parse_complete(napi_env env, napi_status, void *data) {
    auto *j = static_cast<ParseJob *>(data);
    if (j->status != LVBH_OK) {
        napi_value msg, err;
        napi_create_string_utf8(env, j->error.c_str(), NAPI_AUTO_LENGTH, &msg);
        napi_create_error(env, nullptr, msg, &err);
        napi_reject_deferred(env, j->deferred, err);
    } else {
        napi_value out, ab, arr, num, bounds, mn, mx, v;
        void *p = nullptr;
        napi_create_object(env, &out);
        napi_create_arraybuffer(env, j->tri.size() * sizeof(float), &p, &ab);
        if (!j->tri.empty()) std::memcpy(p, j->tri.data(), j->tri.size() * sizeof(float));
        napi_create_typedarray(env, napi_float32_array, j->tri.size(), ab, 0, &arr);
        napi_create_uint32(env, j->n, &num);
        napi_create_object(env, &bounds);
        napi_create_array_with_length(env, 3, &mn);
        napi_create_array_with_length(env, 3, &mx);
        for (uint32_t a = 0; a < 3; ++a) {
            napi_create_double(env, j->bounds[a], &v);
            napi_set_element(env, mn, a, v);
            napi_create_double(env, j->bounds[3 + a], &v);
            napi_set_element(env, mx, a, v);
        }
        napi_set_named_property(env, bounds, "min", mn);
        napi_set_named_property(env, bounds, "max", mx);
        napi_set_named_property(env, out, "NUM_TRIS", num);
        napi_set_named_property(env, out, "TRI_ARR", arr);
        napi_set_named_property(env, out, "BOUNDS", bounds);
        napi_resolve_deferred(env, j->deferred, out);
    }
    napi_delete_async_work(env, j->work);
    delete j;
}

napi_value parse_obj(napi_env env, napi_callback_info info) {
    size_t argc = 1;
    napi_value argv[1];
    void *data = nullptr;
    NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, nullptr, &data));
    auto *j = new ParseJob();
    j->b = static_cast<Builder *>(data);
    napi_valuetype t = napi_undefined;
    if (argc > 0) napi_typeof(env, argv[0], &t);
    bool is_typed = false, is_ab = false;
    if (argc > 0) {
        napi_is_typedarray(env, argv[0], &is_typed);
        napi_is_arraybuffer(env, argv[0], &is_ab);
    }
    if (t == napi_string) {
        size_t len = 0;
        NAPI_OK(env, napi_get_value_string_utf8(env, argv[0], nullptr, 0, &len));
        j->text.resize(len + 1);
        NAPI_OK(env, napi_get_value_string_utf8(env, argv[0], j->text.data(), len + 1, &len));
        j->text.resize(len);
    } else if (is_typed || is_ab) {
        void *raw = nullptr;
        size_t len = 0;
        if (is_typed) {
            napi_typedarray_type type;
            size_t count = 0;
            NAPI_OK(env, napi_get_typedarray_info(env, argv[0], &type, &count, &raw, nullptr, nullptr));
            len = count;  // a Uint8Array: one byte per element
        } else {
            NAPI_OK(env, napi_get_arraybuffer_info(env, argv[0], &raw, &len));
        }
        j->text.assign(static_cast<char *>(raw), static_cast<char *>(raw) + len);
    } else {
        delete j;
        napi_throw_type_error(env, nullptr, "parseObj expects a string or the file's bytes");
        return nullptr;
    }
    napi_value promise, name;
    NAPI_OK(env, napi_create_promise(env, &j->deferred, &promise));
    napi_create_string_utf8(env, "lvbh.parseObj", NAPI_AUTO_LENGTH, &name);
    NAPI_OK(env, napi_create_async_work(env, nullptr, name, parse_execute, parse_complete, j, &j->work));
    NAPI_OK(env, napi_queue_async_work(env, j->work));
    return promise;
}

// initBVHBuild(device) -> { build, parseObj }
napi_value init_bvh_build(napi_env env, napi_callback_info info) {
    size_t argc = 1;
    napi_value argv[1];
    NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr));
    int32_t dev = 0;
    if (argc > 0) napi_get_value_int32(env, argv[0], &dev);
    auto *b = new Builder();
    lvbh_config cfg;
    std::memset(&cfg, 0, sizeof cfg);
    cfg.device = dev;
    if (lvbh_create(&b->ctx, &cfg) != LVBH_OK) {
        delete b;
        napi_throw_error(env, nullptr, "lvbh_create failed");
        return nullptr;
    }
    napi_value obj, fn;
    NAPI_OK(env, napi_create_object(env, &obj));
    NAPI_OK(env, napi_create_function(env, "build", NAPI_AUTO_LENGTH, build, b, &fn));
    NAPI_OK(env, napi_set_named_property(env, obj, "build", fn));
    NAPI_OK(env, napi_create_function(env, "parseObj", NAPI_AUTO_LENGTH, parse_obj, b, &fn));
    NAPI_OK(env, napi_set_named_property(env, obj, "parseObj", fn));
    NAPI_OK(env, napi_wrap(env, obj, b, finalize_builder, nullptr, nullptr));
    return obj;
}

napi_value init(napi_env env, napi_value exports) {
    napi_value fn;
    napi_create_function(env, "initBVHBuild", NAPI_AUTO_LENGTH, init_bvh_build, nullptr, &fn);
    napi_set_named_property(env, exports, "initBVHBuild", fn);
    return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, init)
