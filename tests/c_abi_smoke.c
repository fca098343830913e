/* A plain C caller of the engine's C ABI (include/vqemps.h), the way a C or C++
 * host -- such as a CUDA-Q NVQIR simulator plugin (the reference's
 * simulator_mps_dist.cu:1371-1643) -- would drive it: create a context, load the
 * circuit (qubits mapped to sites n-1-q, the plugin's order), load a Pauli sum,
 * evaluate energies from host buffers, sample from device buffers, read an error
 * message, destroy. The circuit and Hamiltonian are the two-qubit known answer
 * of the reference's install checks (setup_local_cudaq.sh:3023-3061):
 * E(t) = -0.15 + 0.43 sin t - 0.03 cos t. Prints one line per check and exits
 * with the number of failed checks. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "vqemps.h"

static int failures = 0;

static void check(int ok, const char *what) {
  printf("%s %s\n", ok ? "ok" : "FAIL", what);
  if (!ok) ++failures;
}

int main(void) {
  vqemps_ctx *ctx = NULL;
  check(vqemps_create(0, 16, 0.0, 0.0, &ctx) == VQEMPS_OK && ctx != NULL, "create");
  if (!ctx) return 1;
  /* ry(theta[0]) q0; x q1; cx q0 -> q1 */
  vqemps_op ops[3];
  memset(ops, 0, sizeof(ops));
  ops[0].kind = VQEMPS_RY; ops[0].q0 = 0; ops[0].q1 = -1; ops[0].param = 0; ops[0].angle = 1.0; ops[0].matrix = -1;
  ops[1].kind = VQEMPS_X; ops[1].q0 = 1; ops[1].q1 = -1; ops[1].param = -1; ops[1].matrix = -1;
  ops[2].kind = VQEMPS_CX; ops[2].q0 = 0; ops[2].q1 = 1; ops[2].param = -1; ops[2].matrix = -1;
  check(vqemps_set_circuit(ctx, 2, ops, 3, NULL, 0, VQEMPS_INIT_ZERO, 1) == VQEMPS_OK, "set_circuit site_order 1");
  int P = 0;
  check(vqemps_num_params(ctx, &P) == VQEMPS_OK && P == 1, "num_params");
  /* 0.11 I + sum_k (0.11 + 0.03 k) P_k, P = Z0, Z1, X0X1, Y0Y1, Z0Z1, X1 (qubit-ordered rows) */
  const char words[] = "II" "ZI" "IZ" "XX" "YY" "ZZ" "IX";
  double coeffs[7];
  coeffs[0] = 0.11;
  for (int k = 1; k < 7; ++k) coeffs[k] = 0.11 + 0.03 * k;
  int h = -1;
  check(vqemps_set_hamiltonian(ctx, words, coeffs, 7, &h) == VQEMPS_OK && h >= 0, "set_hamiltonian");
  double theta[4] = {0.37, -1.2, 2.5, 0.0}, energies[4] = {0, 0, 0, 0};
  check(vqemps_energy_batch_host(ctx, h, theta, 4, energies, NULL, NULL) == VQEMPS_OK, "energy_batch_host");
  double worst = 0.0;
  for (int b = 0; b < 4; ++b) {
    const double ref = -0.15 + 0.43 * sin(theta[b]) - 0.03 * cos(theta[b]);
    const double err = fabs(energies[b] - ref);
    if (err > worst) worst = err;
  }
  printf("energies %.15f %.15f %.15f %.15f max_abs_err %.3e\n", energies[0], energies[1], energies[2], energies[3],
         worst);
  check(worst < 1e-10, "closed form to 1e-10");
  /* sampling: device buffers, as a CUDA host would pass them */
  const int shots = 4000;
  double *theta_dev = NULL;
  uint64_t *bits_dev = NULL;
  static uint64_t bits[4000];
  int cuda_ok = cudaMalloc((void **)&theta_dev, sizeof(double)) == cudaSuccess &&
                cudaMalloc((void **)&bits_dev, sizeof(uint64_t) * shots) == cudaSuccess &&
                cudaMemcpy(theta_dev, theta, sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
  check(cuda_ok, "device buffers");
  int ones = 0, bad = 0;
  if (cuda_ok) {
    check(vqemps_sample(ctx, theta_dev, 1, shots, 1234567u, VQEMPS_RNG_SPLITMIX, bits_dev, NULL) == VQEMPS_OK,
          "sample");
    check(cudaMemcpy(bits, bits_dev, sizeof(uint64_t) * shots, cudaMemcpyDeviceToHost) == cudaSuccess, "copy shots");
    for (int s = 0; s < shots; ++s) {
      const int q0 = (int)(bits[s] & 1u), q1 = (int)((bits[s] >> 1) & 1u);
      if (q0 == q1) ++bad;        /* the state is cos(t/2)|q0=0,q1=1> + sin(t/2)|q0=1,q1=0> */
      ones += q0;
    }
  }
  const double p1 = pow(sin(0.5 * theta[0]), 2.0);
  const double sigma = sqrt(p1 * (1.0 - p1) / shots);
  printf("shots q0=1 fraction %.4f expected %.4f (sigma %.4f), impossible outcomes %d\n", (double)ones / shots, p1,
         sigma, bad);
  check(bad == 0 && fabs((double)ones / shots - p1) < 5.0 * sigma, "shot frequencies");
  cudaFree(theta_dev);
  cudaFree(bits_dev);
  /* an invalid Pauli character is refused with a message */
  int h2 = -1;
  const int rc = vqemps_set_hamiltonian(ctx, "ZQ", coeffs, 1, &h2);
  const char *msg = vqemps_last_error(ctx);
  printf("invalid word: status %d, message \"%s\"\n", rc, msg ? msg : "(null)");
  check(rc == VQEMPS_INVALID && msg != NULL && msg[0] != '\0', "last_error after invalid input");
  check(vqemps_destroy(ctx) == VQEMPS_OK, "destroy");
  printf("%s\n", failures == 0 ? "all checks passed" : "some checks failed");
  return failures;
}
