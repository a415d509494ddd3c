/* dpu_host.h -- a host stand-in for the UPMEM DPU runtime, just enough to run
 * the reference's own join kernels (src/dpu/src/join/\*.c) as plain C on the CPU.
 * Test infrastructure of the oracle only: nothing in the product includes it.
 *
 * One process is one DPU launch (the kernels keep file-scope state, which a
 * real DPU reinitialises when its program is loaded):
 *   - tasklets are pthreads; me() is the calling thread's tasklet number;
 *   - MRAM is one host array; the kernels address it with 32-bit offsets from
 *     DPU_MRAM_HEAP_POINTER (0 here), and mram_read / mram_write align the MRAM
 *     address down to 8 bytes as the DPU's DMA engine does (the kernels rely on
 *     that when they read a 4-byte offset at an odd index);
 *   - WRAM is a bump-allocated block mapped below 4 GiB, because the kernels
 *     round-trip WRAM pointers through uint32_t;
 *   - the runtime's mutexes are bytes taken with an atomic test-and-set, its
 *     barriers count arrivals per generation; the kernels' atomic-bit arrays
 *     share one section with room past their ends.
 * The DPU intrinsics and their meaning follow the UPMEM SDK documentation
 * (mram.h, alloc.h, barrier.h, mutex.h, defs.h, perfcounter.h). */
#ifndef DPU_HOST_H
#define DPU_HOST_H

#include <pthread.h>
#include <sched.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

/* address-space qualifiers of the DPU compiler: no meaning on the host */
#define __host
#define __mram_ptr
#define __mram
#define __mram_noinit
/* The DPU keeps __atomic_bit arrays in its atomic register of 256 bits, so an
 * index past an array's end still names an atomic bit (two kernels take bits 49
 * and 50 of a 32-entry array). On the host they go to one section that ends
 * with a 256-byte tail (dpu_host.c), so such an index stays inside it. */
#define __atomic_bit __attribute__((section("dpu_atomic")))
#define __dma_aligned __attribute__((aligned(8)))
#define __noinline __attribute__((noinline))

/* MRAM addresses are offsets into the host MRAM array */
#define DPU_MRAM_HEAP_POINTER 0u

/* defs.h */
extern __thread unsigned dpu_host_tasklet;
static inline unsigned me(void) { return dpu_host_tasklet; }

/* mram.h: addresses arrive as pointers or as 32-bit integers */
void dpu_host_mram_read(uintptr_t mram_addr, uintptr_t wram_addr, uint32_t nbytes);
void dpu_host_mram_write(uintptr_t wram_addr, uintptr_t mram_addr, uint32_t nbytes);
#define mram_read(from, to, n) dpu_host_mram_read((uintptr_t)(from), (uintptr_t)(to), (uint32_t)(n))
#define mram_write(from, to, n) dpu_host_mram_write((uintptr_t)(from), (uintptr_t)(to), (uint32_t)(n))

/* alloc.h */
void *mem_alloc(size_t nbytes);
void mem_reset(void);

/* barrier.h */
typedef struct {
    unsigned count, arrived, generation;
    pthread_mutex_t mu;
    pthread_cond_t cv;
} dpu_host_barrier_t;
#define BARRIER_INIT(name, n) \
    dpu_host_barrier_t name = {(n), 0u, 0u, PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER}
void barrier_wait(dpu_host_barrier_t *b);

/* mutex.h: a mutex is a byte (the kernels' __atomic_bit arrays, or MUTEX_INIT) */
typedef uint8_t *mutex_id_t;
#define MUTEX_INIT(name)              \
    static uint8_t name##_dpu_host_byte; \
    static uint8_t *const name = &name##_dpu_host_byte
static inline void mutex_lock(uint8_t *m) {
    while (__atomic_test_and_set(m, __ATOMIC_ACQUIRE)) sched_yield();
}
static inline void mutex_unlock(uint8_t *m) { __atomic_clear(m, __ATOMIC_RELEASE); }

/* perfcounter.h: no cycle counter on the host */
#define COUNT_CYCLES 0
#define COUNT_INSTRUCTIONS 1
typedef uint64_t perfcounter_t;
static inline perfcounter_t perfcounter_config(int mode, bool reset) {
    (void)mode;
    (void)reset;
    return 0;
}
static inline perfcounter_t perfcounter_get(void) { return 0; }

/* Kernel glue (one file per kernel): the __host arguments from the runner's
 * integer list, and the kernel's results back as integers. */
int dpu_host_set_args(const int64_t *args, int nargs);
int dpu_host_get_results(int64_t *out, int cap);

#endif
