/* talsh-b200: the host-memory pinning helpers of the reference's mem_manager.h
 * (:79-80) that its C++ layer calls (talshxx.hpp pinHostMemory and
 * unpinHostMemory).  The rest of the reference's mem_manager.h -- the Host and
 * device argument buffers and their block allocator -- has no counterpart
 * here: device memory comes from a stream-ordered pool under a byte budget and
 * Host bodies allocated by the library are pinned one by one (talsh.h). */
#ifndef TALSH_B200_MEM_MANAGER_H_
#define TALSH_B200_MEM_MANAGER_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pins caller memory [host_ptr, host_ptr + tsize) for fast transfers to every
 * GPU (reference mem_manager.cpp:1480-1492).  0 on success, 1 on a CUDA error
 * (already registered, no device, ...); the error text is kept for
 * tcLastErrorString. */
int host_mem_register(void *host_ptr, size_t tsize);

/* Unpins memory pinned by host_mem_register (reference mem_manager.cpp:1494-1506).
 * 0 on success, 1 on a CUDA error. */
int host_mem_unregister(void *host_ptr);

#ifdef __cplusplus
}
#endif

#endif /* TALSH_B200_MEM_MANAGER_H_ */
