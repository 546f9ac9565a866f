/* Test infrastructure: the reference decoder declares LDPC_iterations extern
 * (LdpcaDecoder.cpp:30, frame.cpp:10) but defines it only in its CUDA host code
 * (LDPCA_cuda.cu:17).  This definition lets the CPU-only build of the reference
 * link; nothing reads it in ParallelMode 0/1. */
int LDPC_iterations = 0;
