// ref_gpu_harness.cu - test infrastructure: runs the reference's own GPU partition, Bloom and probe
// code, compiled for sm_100a from the reference tree (src/kernel_functions.cu,
// src/vlsplit_hash_kernel.cu, src/bloom.cu), so that the engine's pairs can be compared with the
// pairs the reference's GPU path writes for the same inputs. Nothing of the engine is linked.
//
//   ref_gpu_harness bf0  R.bin S.bin R S P1 P2 pairs.bin
//   ref_gpu_harness bf10 R.bin S.bin R S P1 P2 pairs.bin num_bits num_hashes
//
// bf0 is gpu_main's one-PE order with use_bf = 0: R and S partitioned in two levels
// (partial_jointable_gpu_partition_r_only / _s_only, vlsplit_hash_kernel.cu:224-298), then the
// shared-memory hash probe (partial_jointable_gpu_run_only_s, vlsplit_hash_kernel.cu:300-325, as
// join_executor.cu:320-328 calls it). bf10 is the use_bf = 10 order: R partitioned first, one
// insertKernelPartitioned launch per level-1 partition into that partition's filter segment
// (hash_kernel.cu:670-722, segment sizing hash_kernel.cu:561-565), the S prefilter
// queryAndCompactKernelPartitioned (hash_kernel.cu:935-954), then the survivors partitioned and
// probed as in bf0.
//
// Values are the reference's synthesised payloads, row + 1 for R and row + 100000001 for S
// (hash_kernel.cu:333-335). Prints "COUNT n", "OVERFLOW m" (sub-buckets that took the nested-loop
// path, kernel_functions.cu:341-370) and, for bf10, "SURVIVORS s"; writes the n R values, then the
// n S values (int32) to pairs.bin in the order the reference wrote them.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "common.h"
#include "kernel_functions.h"
#include "vlsplit_hash_kernel.h"
#include "bloom.cuh"

// The reference's launch globals (common.h), with the defaults of hash_kernel.cu:38-43.
int partition_size = 128;
int second_partition_size = 67;
int thread_no = 1024;
int block_no = 31250;
int block_size;
int chunk_size = 1024;

#define CK(x)                                                                                     \
    do {                                                                                          \
        cudaError_t e_ = (x);                                                                     \
        if (e_ != cudaSuccess) {                                                                  \
            fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));                              \
            exit(3);                                                                              \
        }                                                                                         \
    } while (0)

static std::vector<int> read_keys(const char* path, long long n) {
    std::vector<int> v(n);
    FILE* f = fopen(path, "rb");
    if (!f || (long long)fread(v.data(), 4, n, f) != n) {
        fprintf(stderr, "read %s\n", path);
        exit(2);
    }
    fclose(f);
    return v;
}

template <class T>
static T* dev_alloc(long long n) {
    T* d = nullptr;
    CK(cudaMalloc(&d, sizeof(T) * (size_t)(n > 0 ? n : 1)));
    CK(cudaMemset(d, 0, sizeof(T) * (size_t)(n > 0 ? n : 1)));
    return d;
}
template <class T>
static T* dev_copy(const std::vector<T>& h) {
    T* d = dev_alloc<T>((long long)h.size());
    if (!h.empty()) CK(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return d;
}

int main(int argc, char** argv) {
    if (argc < 9) {
        fprintf(stderr, "usage: %s bf0|bf10 R.bin S.bin R S P1 P2 pairs.bin [num_bits num_hashes]\n", argv[0]);
        return 2;
    }
    const std::string mode = argv[1];
    const long long R = atoll(argv[4]), S = atoll(argv[5]);
    partition_size = atoi(argv[6]);
    second_partition_size = atoi(argv[7]);
    const bool bf10 = mode == "bf10";
    if ((mode != "bf0" && !bf10) || (bf10 && argc < 11) || R < 1 || S < 0 || R >= (1LL << 31) ||
        S >= (1LL << 31) || partition_size < 1 || partition_size > PARTITION_MAX || second_partition_size < 1 ||
        second_partition_size > SECOND_PASS_MAX) {
        fprintf(stderr, "bad arguments\n");
        return 2;
    }
    std::vector<int> rk = read_keys(argv[2], R), sk = read_keys(argv[3], S), rv(R), sv(S);
    for (long long i = 0; i < R; ++i) rv[i] = (int)i + 1;
    for (long long i = 0; i < S; ++i) sv[i] = (int)i + 100000001;

    cudaStream_t st;
    CK(cudaStreamCreate(&st));
    int *dr = dev_copy(rk), *drv = dev_copy(rv), *ds = dev_copy(sk), *dsv = dev_copy(sv);
    int *dor = dev_alloc<int>(R), *dorv = dev_alloc<int>(R), *dos = dev_alloc<int>(S), *dosv = dev_alloc<int>(S);
    long long *pa = dev_alloc<long long>(partition_size), *pb = dev_alloc<long long>(partition_size);
    long long *br = dev_alloc<long long>(partition_size), *bs = dev_alloc<long long>(partition_size);
    long long *oa = dev_alloc<long long>(partition_size), *ob = dev_alloc<long long>(partition_size);
    const long long fine = (long long)partition_size * second_partition_size;
    long long *sr = dev_alloc<long long>(fine), *ss = dev_alloc<long long>(fine);
    int *dnum = dev_alloc<int>(1), *widx = dev_alloc<int>(1);

    partial_jointable_gpu_partition_r_only(dr, dor, drv, dorv, pa, br, oa, sr, R, st);
    CK(cudaGetLastError());

    int* s_keys = ds;
    int* s_vals = dsv;
    long long s_n = S;
    if (bf10) {
        const size_t num_bits = (size_t)atoll(argv[9]);
        const int num_hashes = atoi(argv[10]);
        size_t pp_bits = ((num_bits / (size_t)partition_size + 255) / 256) * 256;
        if (pp_bits < 256) pp_bits = 256;
        const size_t pp_words = pp_bits / 32, total_words = pp_words * (size_t)partition_size;
        uint32_t* pbf = dev_alloc<uint32_t>((long long)total_words);
        std::vector<long long> hb(partition_size);
        CK(cudaMemcpy(hb.data(), br, sizeof(long long) * partition_size, cudaMemcpyDeviceToHost));
        const int threads = 256;
        for (int p = 0; p < partition_size; ++p) {
            const long long b = p == 0 ? 0 : hb[p - 1], e = hb[p];
            if (e - b <= 0) continue;
            insertKernelPartitioned<<<(unsigned)((e - b + threads - 1) / threads), threads, 0, st>>>(
                pbf + (size_t)p * pp_words, dr, b, e, num_hashes, pp_bits);
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        int *fs = dev_alloc<int>(S), *fsv = dev_alloc<int>(S);
        long long* cnt = dev_alloc<long long>(1);
        const long long pf_block = S / block_no + (S % block_no != 0);
        if (S > 0) {
            queryAndCompactKernelPartitioned<<<block_no, thread_no>>>(pbf, ds, dsv, (int)S, num_hashes, pp_bits, pp_words,
                                                                      partition_size, fs, fsv, cnt, (int)pf_block);
            CK(cudaGetLastError());
            CK(cudaDeviceSynchronize());
            CK(cudaMemcpy(&s_n, cnt, sizeof(long long), cudaMemcpyDeviceToHost));
        } else {
            s_n = 0;
        }
        printf("SURVIVORS %lld\n", s_n);
        s_keys = fs;
        s_vals = fsv;
    }
    partial_jointable_gpu_partition_s_only(s_keys, dos, s_vals, dosv, nullptr, pb, bs, ob, ss, dnum, s_n, st);
    CK(cudaGetLastError());

    const long long cap = s_n + 16;
    int *ans = dev_alloc<int>(cap), *ansv = dev_alloc<int>(cap), *anss = dev_alloc<int>(cap);
    const int capi = (int)cap, zero = 0;
    CK(cudaMemcpyToSymbol(d_answer_capacity, &capi, sizeof(int)));
    CK(cudaMemcpyToSymbol(d_probe_overflow_count, &zero, sizeof(int)));
    int count = -1;
    partial_jointable_gpu_run_only_s(dr, s_keys, drv, s_vals, br, bs, sr, ss, ans, ansv, anss, dnum, HT_SIZE + 1, &count,
                                     st, nullptr, widx);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    int overflow = 0;
    CK(cudaMemcpyFromSymbol(&overflow, d_probe_overflow_count, sizeof(int)));
    printf("COUNT %d\nOVERFLOW %d\n", count, overflow);
    if (count < 0 || count > cap) return 1;
    std::vector<int> a(count), b(count);
    if (count) {
        CK(cudaMemcpy(a.data(), ansv, sizeof(int) * count, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(b.data(), anss, sizeof(int) * count, cudaMemcpyDeviceToHost));
    }
    FILE* f = fopen(argv[8], "wb");
    if (!f) return 2;
    fwrite(a.data(), 4, a.size(), f);
    fwrite(b.data(), 4, b.size(), f);
    fclose(f);
    return 0;
}
