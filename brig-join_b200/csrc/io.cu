// io.cu - the reference's file formats at the boundary (host code only).
//
// Inputs: one relation per file, headerless little-endian int32: the n keys, followed by the n
// values when the file carries them (datagen/gen_dataset.cpp writes the key block; gpu_main reads
// it, and the value block after it with --read_val 1, src/hash_kernel.cu:300-335). Without values
// the reference synthesises row + 1 for R and row + 100000001 for S.
// Outputs: the reference parses an output path and never writes it (src/driver.cpp:50,119); the
// engine writes the pairs in the same headerless block layout as its inputs: keys (optional), then R
// values, then S values.
#include <cstdio>
#include "../../include/brig_join.h"
#include "engine.h"

extern "C" int brig_join_read_relation(const char* path, int64_t n, int32_t read_val, uint32_t val_base,
                                       uint32_t* keys, uint32_t* vals) {
    using namespace brig;
    try {
        if (!path || n < 0 || (n > 0 && !keys) || (read_val && n > 0 && !vals))
            fail(BRIG_E_INVALID, "brig_join_read_relation: bad argument");
        FILE* f = std::fopen(path, "rb");
        if (!f) fail(BRIG_E_INVALID, std::string("cannot open ") + path);
        const size_t got_k = n > 0 ? std::fread(keys, 4, (size_t)n, f) : 0;
        const size_t got_v = (read_val && n > 0) ? std::fread(vals, 4, (size_t)n, f) : (size_t)n;
        std::fclose(f);
        if (got_k != (size_t)n || got_v != (size_t)n)
            fail(BRIG_E_INVALID, std::string(path) + " is shorter than " + std::to_string(n) +
                                     (read_val ? " keys and values" : " keys"));
        if (!read_val && vals)
            for (int64_t i = 0; i < n; ++i) vals[i] = val_base + (uint32_t)i;
        return BRIG_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.status;
    }
}

extern "C" int brig_join_write_pairs(const char* path, const uint32_t* key, const uint32_t* r_val,
                                     const uint32_t* s_val, int64_t n) {
    using namespace brig;
    try {
        if (!path || n < 0 || (n > 0 && (!r_val || !s_val))) fail(BRIG_E_INVALID, "brig_join_write_pairs: bad argument");
        FILE* f = std::fopen(path, "wb");
        if (!f) fail(BRIG_E_INVALID, std::string("cannot create ") + path);
        bool ok = true;
        if (n > 0) {
            if (key) ok = ok && std::fwrite(key, 4, (size_t)n, f) == (size_t)n;
            ok = ok && std::fwrite(r_val, 4, (size_t)n, f) == (size_t)n;
            ok = ok && std::fwrite(s_val, 4, (size_t)n, f) == (size_t)n;
        }
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) fail(BRIG_E_INVALID, std::string("write to ") + path + " failed");
        return BRIG_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.status;
    }
}
