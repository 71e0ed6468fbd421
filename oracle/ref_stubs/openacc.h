/* Host-only stand-in for the OpenACC runtime header, used when the
 * reference's particles.c / neighbors.c are compiled with plain gcc: the
 * `#pragma acc` lines are ignored and every loop runs serially on the host.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref build). */
#ifndef SPHPC_ORACLE_OPENACC_STUB_H_
#define SPHPC_ORACLE_OPENACC_STUB_H_
#define acc_async_sync (-1)
void *acc_get_cuda_stream(int async);
#endif
