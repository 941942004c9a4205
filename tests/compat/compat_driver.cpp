// compat_driver.cpp - calls the engine through the reference-named C++ entry points
// (include/brig_join_compat.h), the way BRIG-Join's own host code would.
//   compat_driver gpu_main R.bin S.bin R S use_bf            -> prints the reference's total line
//   compat_driver parts    R.bin S.bin R S P1 P2 pairs.bin    -> partition R and S, check the
//                                                                reference layout, probe, dump pairs
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

int main(int argc, char** argv) {
    if (argc < 6) return 2;
    const std::string mode = argv[1];
    const long long R = atoll(argv[4]), S = atoll(argv[5]);
    if (mode == "gpu_main") {
        gpu_main(nullptr, nullptr, argv[2], argv[3], R, S, atoi(argv[6]), false, false, 0.1, 2);
        return 0;
    }
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
    partial_jointable_gpu_run_only_s(da, db, dav, dbv, br, bs, sr, ss, ans, ansv, anss, dnum, 10008, &count, 0, nullptr,
                                     widx);
    printf("COUNT %d\n", count);
    std::vector<int> a = host(ansv, count > 0 ? count : 0), b = host(anss, count > 0 ? count : 0);
    FILE* f = fopen(argv[8], "wb");
    fwrite(a.data(), 4, a.size(), f);
    fwrite(b.data(), 4, b.size(), f);
    fclose(f);
    return lay ? 0 : 1;
}
