/*
 * C ABI of the learned warm start's message-passing network (forward,
 * backward, loss and Adam on one CUDA device).
 *
 * No reference counterpart: the reference initialises its global VQE from the
 * plain partition warm start (test/sources/independent-vqe/Qiskit_VQE/
 * independent_vqe.py:257-305, local solves mapped by layer/qubit/gate). The
 * network proposes the same angle vector directly from the Hamiltonian's
 * qubit-coupling graph; the engine's exact MPS energy judges the proposal and
 * the partition warm start remains the fallback.
 *
 * All device pointers are caller-owned (torch tensors); every call is ordered
 * on the given stream; weights are FP32 master copies rounded to BF16 at every
 * matrix product (FP32 accumulation).
 */
#ifndef VQEMPS_MPNN_ABI_H
#define VQEMPS_MPNN_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum vqemps_mpnn_status {
  VQEMPS_MPNN_OK = 0,
  VQEMPS_MPNN_INVALID = 3,
  VQEMPS_MPNN_CUDA_ERROR = 4
};

typedef struct vqemps_mpnn vqemps_mpnn;

/* A batch of graphs as one graph in device memory. Edges are directed and
 * sorted by destination: edges into node i are dst_off[i] .. dst_off[i+1).
 * src_perm lists the edge ids sorted by source, src_off its offsets. */
typedef struct vqemps_graph {
  int32_t num_nodes, num_edges;
  const float *node_feat;   /* num_nodes x node_in */
  const float *edge_feat;   /* num_edges x edge_in */
  const int32_t *edge_src;  /* num_edges */
  const int32_t *edge_dst;  /* num_edges */
  const int32_t *dst_off;   /* num_nodes + 1 */
  const int32_t *src_perm;  /* num_edges */
  const int32_t *src_off;   /* num_nodes + 1 */
} vqemps_graph;

/* width: a multiple of 16, at most 128; layers <= 7; out_per_node angles per
 * node. Parameters start at zero: load them with vqemps_mpnn_set_params. */
int vqemps_mpnn_create(int device, int node_in, int edge_in, int width, int layers, int out_per_node,
                       vqemps_mpnn **out);
int vqemps_mpnn_destroy(vqemps_mpnn *net);
const char *vqemps_mpnn_last_error(const vqemps_mpnn *net);
/* Flat parameter vector: Win [node_in x W], bin [W]; per layer Wm [(W + edge_in)
 * x W], bm [W], Wu [2W x W], bu [W]; Wo [W x out], bo [out] (row-major, rows =
 * inputs). set_params also resets the Adam state. */
int vqemps_mpnn_num_params(const vqemps_mpnn *net, int64_t *count);
int vqemps_mpnn_set_params(vqemps_mpnn *net, const float *host, int64_t count);
int vqemps_mpnn_get_params(vqemps_mpnn *net, float *host, int64_t count);
/* angles_dev (may be NULL): num_nodes x out_per_node, theta = pi tanh(z).
 * Keeps the activations for loss / backward on the same graph. */
int vqemps_mpnn_forward(vqemps_mpnn *net, const vqemps_graph *graph, float *angles_dev, void *stream);
/* Periodic angle loss of the last forward: sum_i w_i sum_j (1 - cos(theta_ij -
 * target_ij)) / (out * sum_i w_i); node_weight_dev may be NULL (all 1);
 * loss_dev (1 float) and dangles_dev (its gradient) may be NULL. */
int vqemps_mpnn_loss(vqemps_mpnn *net, const float *target_dev, const float *node_weight_dev, float *loss_dev,
                     float *dangles_dev, void *stream);
/* grad_dev (num_params floats, overwritten) = d(sum dangles * angles)/d(params)
 * through the last forward. */
int vqemps_mpnn_backward(vqemps_mpnn *net, const vqemps_graph *graph, const float *dangles_dev, float *grad_dev,
                         void *stream);
/* One Adam step on the master weights (bias-corrected; weight_decay is L2). */
int vqemps_mpnn_adam_step(vqemps_mpnn *net, const float *grad_dev, float lr, float beta1, float beta2, float eps,
                          float weight_decay, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* VQEMPS_MPNN_ABI_H */
