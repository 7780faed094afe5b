// Host-side state behind an he_handle.
#pragma once
#include <vector>

#include "common.cuh"

struct he_operator {
    int device = 0;
    int n = 0, nc = 0, nt = 0, nv = 0, nd = 0, nlam = 0;
    bool separable = false;
    bool has32 = false;
    he::DeviceTables<double> t64{};
    he::DeviceTables<float> t32{};
    const double2 *tdiag = nullptr;     // diagonal of the kinetic CSR (n entries)
    std::vector<void *> allocations;    // every cudaMalloc made for this handle
    ~he_operator();
};

int he_fail(int status, const char *what, const char *file, int line);
