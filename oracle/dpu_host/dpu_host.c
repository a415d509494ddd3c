/* dpu_host.c -- runtime and runner of the host stand-in for the DPU runtime
 * (dpu_host.h). Test infrastructure of the oracle only.
 *
 * A runner executable is one reference kernel (its main renamed
 * dpu_kernel_main), this file and the kernel's glue. One run is one DPU launch:
 *   stdin:  int64 ntasklets, int64 nargs, int64 args[nargs],
 *           int64 mram_bytes, mram_bytes bytes (the DPU's MRAM image)
 *   stdout: int64 status (0, or the error below), int64 nres, int64 res[nres],
 *           int64 mram_bytes, the MRAM image after the launch
 * status: 1 bad input, 2 an MRAM access outside the image, 3 WRAM exhausted. */
#define _GNU_SOURCE
#include "dpu_host.h"

#include <stdio.h>
#include <stdlib.h>
#include <sys/mman.h>

int dpu_kernel_main(void);

__thread unsigned dpu_host_tasklet;

/* Room past the kernel's atomic-bit array (linked before this file, so it comes
 * first in the section): the DPU's atomic register has 256 bits. */
__attribute__((section("dpu_atomic"), used)) uint8_t dpu_host_atomic_tail[256];

static uint8_t *g_mram;
static uint64_t g_mram_bytes;
static uint8_t *g_wram;
static const uint64_t kWramBytes = 1u << 20;  /* the DPU has 64 KiB; headroom costs nothing */
static uint64_t g_wram_used;
static int g_status;

void dpu_host_mram_read(uintptr_t mram_addr, uintptr_t wram_addr, uint32_t nbytes) {
    const uint64_t a = (uint64_t)mram_addr & ~(uint64_t)7;
    if (a + nbytes > g_mram_bytes) {
        __atomic_store_n(&g_status, 2, __ATOMIC_RELAXED);
        return;
    }
    memcpy((void *)wram_addr, g_mram + a, nbytes);
}

void dpu_host_mram_write(uintptr_t wram_addr, uintptr_t mram_addr, uint32_t nbytes) {
    const uint64_t a = (uint64_t)mram_addr & ~(uint64_t)7;
    if (a + nbytes > g_mram_bytes) {
        __atomic_store_n(&g_status, 2, __ATOMIC_RELAXED);
        return;
    }
    memcpy(g_mram + a, (const void *)wram_addr, nbytes);
}

void *mem_alloc(size_t nbytes) {
    const uint64_t n = ((uint64_t)nbytes + 7) & ~(uint64_t)7;
    const uint64_t at = __atomic_fetch_add(&g_wram_used, n, __ATOMIC_RELAXED);
    if (at + n > kWramBytes) {
        __atomic_store_n(&g_status, 3, __ATOMIC_RELAXED);
        return g_wram; /* the run is reported as failed */
    }
    return g_wram + at;
}

void mem_reset(void) { __atomic_store_n(&g_wram_used, 0, __ATOMIC_RELAXED); }

void barrier_wait(dpu_host_barrier_t *b) {
    pthread_mutex_lock(&b->mu);
    const unsigned gen = b->generation;
    if (++b->arrived == b->count) {
        b->arrived = 0;
        b->generation++;
        pthread_cond_broadcast(&b->cv);
    } else {
        while (gen == b->generation) pthread_cond_wait(&b->cv, &b->mu);
    }
    pthread_mutex_unlock(&b->mu);
}

static void *tasklet(void *arg) {
    dpu_host_tasklet = (unsigned)(uintptr_t)arg;
    dpu_kernel_main();
    return NULL;
}

static int read_all(void *p, size_t n) { return fread(p, 1, n, stdin) == n ? 0 : -1; }
static void write_all(const void *p, size_t n) { fwrite(p, 1, n, stdout); }

int main(void) {
    int64_t ntasklets = 0, nargs = 0, mram_bytes = 0;
    int64_t args[64];
    if (read_all(&ntasklets, 8) || read_all(&nargs, 8) || nargs < 0 || nargs > 64 ||
        read_all(args, (size_t)nargs * 8) || read_all(&mram_bytes, 8) || ntasklets < 1 || ntasklets > 24 ||
        mram_bytes < 8 || mram_bytes > ((int64_t)1 << 32))
        g_status = 1;
    if (!g_status) {
        g_mram_bytes = (uint64_t)mram_bytes;
        g_mram = (uint8_t *)malloc((size_t)g_mram_bytes);
        /* WRAM below 4 GiB: the kernels keep WRAM addresses in uint32_t */
        void *w = mmap(NULL, kWramBytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_32BIT, -1, 0);
        g_wram = w == MAP_FAILED ? NULL : (uint8_t *)w;
        if (!g_mram || !g_wram || read_all(g_mram, (size_t)g_mram_bytes) || dpu_host_set_args(args, (int)nargs))
            g_status = 1;
    }
    if (!g_status) {
        pthread_t th[24];
        for (int64_t t = 0; t < ntasklets; t++) pthread_create(&th[t], NULL, tasklet, (void *)(uintptr_t)t);
        for (int64_t t = 0; t < ntasklets; t++) pthread_join(th[t], NULL);
    }
    /* the kernels print progress lines on stdout: the binary reply follows a marker */
    fflush(stdout);
    const char marker[8] = {'D', 'P', 'U', 'H', 'O', 'S', 'T', '\n'};
    write_all(marker, 8);
    int64_t res[64];
    const int64_t nres = g_status ? 0 : dpu_host_get_results(res, 64);
    const int64_t status = g_status;
    write_all(&status, 8);
    write_all(&nres, 8);
    write_all(res, (size_t)nres * 8);
    const int64_t out_bytes = g_status ? 0 : (int64_t)g_mram_bytes;
    write_all(&out_bytes, 8);
    if (out_bytes) write_all(g_mram, (size_t)out_bytes);
    fflush(stdout);
    return 0;
}
