// compat_driver.cpp - calls the engine through the reference-named C++ entry points
// (include/brig_join_compat.h), the way BRIG-Join's own host code would.
//   compat_driver gpu_main R.bin S.bin R S use_bf            -> prints the reference's total line
//   compat_driver parts    R.bin S.bin R S P1 P2 pairs.bin    -> partition R and S, check the
//                                                                reference layout, probe, dump pairs
//   compat_driver exec     R.bin S.bin R S P1 P2 pairs.bin    -> the same probe through
//                                                                join_execute_host and a JoinChunkContext
//   compat_driver bloom    R.bin S.bin R S bits hashes        -> BloomFilter built from R's keys:
//                                                                every bit where the reference puts it
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "brig_join_compat.h"

static std::vector<int> read_keys(const char* path, long long n) {
    std::vector<int> v(n);
    FILE* f = fopen(path, "rb");
    if (!f || (long long)fread(v.data(), 4, n, f) != n) { fprintf(stderr, "read %s\n", path); exit(2); }
    fclose(f);
    return v;
}

template <class T> static T* dev(const std::vector<T>& h) {
    T* d = nullptr;
    cudaMalloc(&d, sizeof(T) * (h.size() ? h.size() : 1));
    if (!h.empty()) cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    return d;
}
template <class T> static std::vector<T> host(const T* d, size_t n) {
    std::vector<T> h(n);
    if (n) cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost);
    return h;
}

// Every key sits in the bucket and sub-bucket its indexes say: (unsigned)key % P1, then % P2.
static bool check_layout(const std::vector<int>& keys, const std::vector<long long>& blk,
                         const std::vector<long long>& sec, int P1, int P2) {
    long long start = 0;
    for (int p = 0; p < P1; ++p) {
        long long sub = start;
        for (int q = 0; q < P2; ++q) {
            const long long end = start + sec[(size_t)p * P2 + q];
            for (long long i = sub; i < end; ++i)
                if ((unsigned)keys[i] % (unsigned)P1 != (unsigned)p || (unsigned)keys[i] % (unsigned)P2 != (unsigned)q)
                    return false;
            sub = end;
        }
        if (sub != blk[p]) return false;
        start = blk[p];
    }
    return start == (long long)keys.size();
}

// The reference's Bloom hash and bit placement (src/bloom.cu:24-31,153-190), restated on the host:
// block hash(v, 1) % blocks, bit hash(v, i + 1) % 256 of the block for i < k.
static uint32_t ref_hash(int v, uint32_t seed) {
    uint32_t h = seed ^ (uint32_t)v;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// Builds a BloomFilter from R's keys on the device and checks its words against the host
// restatement bit for bit, then that every R key passes and the S keys that pass on the device are
// exactly those that pass on the host.
static int bloom_check(const char* rf, const char* sf, long long R, long long S, long long bits, int k) {
    std::vector<int> rk = read_keys(rf, R), sk = read_keys(sf, S);
    int *dr = dev(rk), *ds = dev(sk);
    BloomFilter bf((size_t)bits, k);
    bf.buildFromTable(dr, (size_t)R);
    const size_t words = bf.getNumWords(), blocks = bf.getNumBits() / 256;
    std::vector<uint32_t> got = host(bf.getDeviceFilter(), words), want(words, 0u);
    for (long long i = 0; i < R; ++i) {
        const size_t b = ref_hash(rk[i], 1u) % blocks;
        for (int j = 0; j < k; ++j) {
            const uint32_t pos = ref_hash(rk[i], (uint32_t)j + 1u) % 256u;
            want[b * 8 + pos / 32] |= 1u << (pos % 32);
        }
    }
    const bool same = got == want;
    long long host_pass = 0;
    for (long long i = 0; i < S; ++i) {
        const size_t b = ref_hash(sk[i], 1u) % blocks;
        bool ok = true;
        for (int j = 0; j < k; ++j) {
            const uint32_t pos = ref_hash(sk[i], (uint32_t)j + 1u) % 256u;
            ok = ok && (want[b * 8 + pos / 32] >> (pos % 32) & 1u);
        }
        host_pass += ok;
    }
    const long long r_pass = bf.query(dr, (size_t)R, nullptr), s_pass = bf.query(ds, (size_t)S, nullptr);
    printf("BLOOM words %zu same %d r_pass %lld s_pass %lld host_s_pass %lld\n", words, same ? 1 : 0, r_pass, s_pass,
           host_pass);
    return (same && r_pass == R && s_pass == host_pass) ? 0 : 1;
}

int main(int argc, char** argv) {
    if (argc < 6) return 2;
    const std::string mode = argv[1];
    const long long R = atoll(argv[4]), S = atoll(argv[5]);
    if (mode == "gpu_main") {
        gpu_main(nullptr, nullptr, argv[2], argv[3], R, S, atoi(argv[6]), false, false, 0.1, 2);
        return 0;
    }
    if (mode == "bloom") return bloom_check(argv[2], argv[3], R, S, atoll(argv[6]), atoi(argv[7]));
    const int P1 = atoi(argv[6]), P2 = atoi(argv[7]);
    partition_size = P1;
    second_partition_size = P2;
    std::vector<int> rk = read_keys(argv[2], R), sk = read_keys(argv[3], S), rv(R), sv(S);
    for (long long i = 0; i < R; ++i) rv[i] = (int)i + 1;
    for (long long i = 0; i < S; ++i) sv[i] = (int)i + 100000001;
    int *da = dev(rk), *dav = dev(rv), *db = dev(sk), *dbv = dev(sv);
    int *doa = dev(std::vector<int>(R)), *doav = dev(std::vector<int>(R));
    int *dob = dev(std::vector<int>(S)), *dobv = dev(std::vector<int>(S));
    std::vector<long long> zP1(P1), zF((size_t)P1 * P2);
    long long *pa = dev(zP1), *pb = dev(zP1), *br = dev(zP1), *bs = dev(zP1), *oa = dev(zP1), *ob = dev(zP1);
    long long *sr = dev(zF), *ss = dev(zF);
    int* dnum = dev(std::vector<int>(1));
    int* widx = dev(std::vector<int>(1));
    int2* kv = nullptr;
    cudaMalloc(&kv, 8 * (S ? S : 1));
    partial_jointable_gpu_partition_r_only(da, doa, dav, doav, pa, br, oa, sr, R, 0);
    partial_jointable_gpu_partition_s_only(db, dob, dbv, dobv, kv, pb, bs, ob, ss, dnum, S, 0);
    const bool lay = check_layout(host(da, R), host(br, P1), host(sr, zF.size()), P1, P2) &&
                     check_layout(host(db, S), host(bs, P1), host(ss, zF.size()), P1, P2);
    printf("LAYOUT %s\n", lay ? "OK" : "BAD");
    const long long cap = S + 16;
    int *ans = dev(std::vector<int>(cap)), *ansv = dev(std::vector<int>(cap)), *anss = dev(std::vector<int>(cap));
    brig_compat_set_answer_capacity(cap);
    int count = -1;
    if (mode == "exec") {
        // one PE: R and S partitioned in place above, their indexes in the context
        JoinChunkContext ctx;
        std::memset(&ctx, 0, sizeof(ctx));
        long long* s_block[1] = {bs};
        long long* s_second[1] = {ss};
        int host_num = 0, total = 0, overflow = 0;
        double probe_sec = 0.0;
        ctx.me = 0;
        ctx.device_num = 1;
        ctx.use_bf = 10;
        ctx.kernel_fusion = 1;
        ctx.GPUA_split = da;
        ctx.GPUA_val_split = dav;
        ctx.GPU_block_index_split_R = br;
        ctx.GPU_block_index_split_S = s_block;
        ctx.GPU_second_index_split_R = sr;
        ctx.GPU_second_index_split_S = s_second;
        ctx.GPU_answer = ans;
        ctx.GPU_answer_val = ansv;
        ctx.GPU_answer_s_val = anss;
        ctx.GPU_answer_num = dnum;
        ctx.GPU_answer_write_idx = widx;
        ctx.answer_num_host = &host_num;
        ctx.max_int_number_for_shared_memory = 10008;
        ctx.first_pass_probe_sec = &probe_sec;
        ctx.total_answer_num = &total;
        ctx.total_overflow_count = &overflow;
        join_execute_host(ctx, db, dbv, S);
        count = total;
        printf("EXEC host_num %d overflow %d\n", host_num, overflow);
        if (host_num != total || overflow != 0) return 1;
    } else {
        partial_jointable_gpu_run_only_s(da, db, dav, dbv, br, bs, sr, ss, ans, ansv, anss, dnum, 10008, &count, 0,
                                         nullptr, widx);
    }
    printf("COUNT %d\n", count);
    std::vector<int> a = host(ansv, count > 0 ? count : 0), b = host(anss, count > 0 ? count : 0);
    FILE* f = fopen(argv[8], "wb");
    fwrite(a.data(), 4, a.size(), f);
    fwrite(b.data(), 4, b.size(), f);
    fclose(f);
    return lay ? 0 : 1;
}
