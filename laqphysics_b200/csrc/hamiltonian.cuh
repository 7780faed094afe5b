// Launchers of the H·psi kernel family (hamiltonian.cu).
#pragma once
#include "common.cuh"

namespace he {

template <typename R>
int launch_hpsi(const DeviceTables<R> &t, const cplx<R> *psi, cplx<R> *out, const double *field, int velocity,
                cplx<R> beta, cplx<R> gamma, cudaStream_t stream);

int launch_diagonal(const DeviceTables<double> &t, const double2 *tdiag, double2 *out, cudaStream_t stream);

}  // namespace he
