// ref_harness.cpp - calls the reference's own CPU join, run_sanity_check (src/sanity_check.cpp,
// compiled from the reference sources by oracle/Makefile into oracle/_ref/). The reference prints
// its count instead of returning it (src/sanity_check.cpp:65), so the harness redirects stdout to
// a temporary file around the call and parses "Answer Num (hash-based): N". Test and baseline
// infrastructure only.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fcntl.h>
#include <omp.h>
#include <string>
#include <unistd.h>

#include "sanity_check.h"

extern "C" long long ref_sanity_count(const int* R, long long nR, const int* S, long long nS, double* seconds) {
    if (nR <= 0 || nS <= 0) {
        if (seconds) *seconds = 0.0;
        return 0;
    }
    fflush(stdout);
    char path[] = "/tmp/brig_ref_sanity_XXXXXX";
    const int fd = mkstemp(path);
    if (fd < 0) return -1;
    const int saved = dup(1);
    dup2(fd, 1);
    const auto t0 = std::chrono::steady_clock::now();
    run_sanity_check(R, nR, S, nS);
    const auto t1 = std::chrono::steady_clock::now();
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    std::string text;
    lseek(fd, 0, SEEK_SET);
    char buf[4096];
    ssize_t k;
    while ((k = read(fd, buf, sizeof(buf))) > 0) text.append(buf, (size_t)k);
    close(fd);
    unlink(path);
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    const char* tag = "Answer Num (hash-based): ";
    const size_t at = text.find(tag);
    if (at == std::string::npos) return -1;
    return std::strtoll(text.c_str() + at + std::strlen(tag), nullptr, 10);
}

extern "C" int ref_omp_max_threads(void) { return omp_get_max_threads(); }
