// ref_cpu_shim.cpp -- C entry point around the reference's CPU split
// (src/cpu_scan.h:20-50), compiled from the reference tree as it lies.
// TEST INFRASTRUCTURE ONLY: used to pin the oracle, never by the product.
#include <cstdlib>
#include "cpu_scan.h"

extern "C" void ref_cpu_split_f32(float* total, int n, float pivot, int* n_slow, int* n_fast) {
    partition_c sizes{0, 0};
    cpu_split<float>(total, nullptr, nullptr, pivot, &sizes, n);
    *n_slow = sizes.N_slow;
    *n_fast = sizes.N_fast;
}

extern "C" void ref_cpu_split_f64(double* total, int n, double pivot, int* n_slow, int* n_fast) {
    partition_c sizes{0, 0};
    cpu_split<double>(total, nullptr, nullptr, pivot, &sizes, n);
    *n_slow = sizes.N_slow;
    *n_fast = sizes.N_fast;
}
