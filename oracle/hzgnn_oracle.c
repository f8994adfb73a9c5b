/*
 * hzgnn_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU oracle for the learned
 * smoother-weight network (forward and backward).  Filled in with the GNN.
 */
int or_gnn_version(void) { return 0; }
