/*
 * CPU restatement of the reference's CPU energy path -- TEST INFRASTRUCTURE ONLY
 * (the timed CPU baseline of bench.py and a checker in tests; never the product).
 *
 * Restates ReverseMPS.energy_chunk (test/tools/reverse_mps.py:59-82) on the exact
 * bond-doubling MPS (reverse_mps.py:39-57): the Hamiltonian is processed in
 * chunks of `chunk` terms in input order; within a chunk, words sharing a prefix
 * share environments (one node per distinct (parent, Pauli) per site); every node
 * applies E' = sum_{i,i'} conj(A[a,i,b]) P[i,i'] E[a,a'] A[a',i',c]; the value of
 * a word is Re E[0,0] after the last site. Complex128 throughout. Chunks run in
 * parallel on OpenMP threads (the reference runs them sequentially on torch).
 */
#include <complex.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define CHI 16
typedef double complex cd;

static int code_of(char c) { return c == 'X' ? 1 : c == 'Y' ? 2 : c == 'Z' ? 3 : 0; }

/* E' for one node. A: site tensor [CHI][2][CHI], dims dl x 2 x dr. */
static void transfer(const cd *E, const cd *A, int p, int dl, int dr, cd *out, cd *tmp) {
  /* tmp[a][i][c] = sign_i * sum_a' E[a][a'] A[a'][flip(i)][c] */
  for (int a = 0; a < dl; ++a)
    for (int i = 0; i < 2; ++i) {
      const int ip = (p == 1 || p == 2) ? 1 - i : i;
      cd sign = 1.0;
      if (p == 3 && i == 1) sign = -1.0;
      if (p == 2) sign = i ? I : -I;
      for (int c = 0; c < dr; ++c) {
        cd acc = 0.0;
        for (int k = 0; k < dl; ++k) acc += E[a * CHI + k] * A[(k * 2 + ip) * CHI + c];
        tmp[(a * 2 + i) * CHI + c] = sign * acc;
      }
    }
  for (int b = 0; b < dr; ++b)
    for (int c = 0; c < dr; ++c) {
      cd acc = 0.0;
      for (int a = 0; a < dl; ++a)
        for (int i = 0; i < 2; ++i) acc += conj(A[(a * 2 + i) * CHI + b]) * tmp[(a * 2 + i) * CHI + c];
      out[b * CHI + c] = acc;
    }
}

/* sites: n padded tensors (re, im interleaved); dims: n + 1 bond dims;
 * words: T rows of n chars (site order); returns sum_k c_k Re<P_k>. */
double cpu_energy(int n, const double *sites, const int *dims, const char *words, const double *coeffs,
                  int T, int chunk, int threads) {
  const cd *A = (const cd *)sites;
  const int nchunks = (T + chunk - 1) / chunk;
  double total = 0.0;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(+ : total)
  {
    cd *e0 = malloc(sizeof(cd) * chunk * CHI * CHI);
    cd *e1 = malloc(sizeof(cd) * chunk * CHI * CHI);
    cd *tmp = malloc(sizeof(cd) * CHI * 2 * CHI);
    int *prev = malloc(sizeof(int) * chunk), *cur = malloc(sizeof(int) * chunk);
    int *parents = malloc(sizeof(int) * chunk), *pauli = malloc(sizeof(int) * chunk);
    int *table = malloc(sizeof(int) * chunk * 4);
#pragma omp for schedule(dynamic)
    for (int ch = 0; ch < nchunks; ++ch) {
      const int t0 = ch * chunk;
      const int cnt = T - t0 < chunk ? T - t0 : chunk;
      cd *ein = e0, *eout = e1;
      memset(ein, 0, sizeof(cd) * CHI * CHI);
      ein[0] = 1.0;
      int nprev = 1;
      for (int j = 0; j < cnt; ++j) prev[j] = 0;
      for (int q = 0; q < n; ++q) {
        for (int k = 0; k < nprev * 4; ++k) table[k] = -1;
        int nodes = 0;
        for (int j = 0; j < cnt; ++j) {
          const int key = prev[j] * 4 + code_of(words[(size_t)(t0 + j) * n + q]);
          if (table[key] < 0) {
            table[key] = nodes;
            parents[nodes] = prev[j];
            pauli[nodes] = key & 3;
            ++nodes;
          }
          cur[j] = table[key];
        }
        const cd *Aq = A + (size_t)q * CHI * 2 * CHI;
        for (int k = 0; k < nodes; ++k)
          transfer(ein + (size_t)parents[k] * CHI * CHI, Aq, pauli[k], dims[q], dims[q + 1],
                   eout + (size_t)k * CHI * CHI, tmp);
        cd *t = ein; ein = eout; eout = t;
        int *u = prev; prev = cur; cur = u;
        nprev = nodes;
      }
      for (int j = 0; j < cnt; ++j) total += coeffs[t0 + j] * creal(ein[(size_t)prev[j] * CHI * CHI]);
    }
    free(e0); free(e1); free(tmp); free(prev); free(cur); free(parents); free(pauli); free(table);
  }
  return total;
}
