/* Empty stand-in for the UPMEM DPU runtime header <mutex.h>. The reference's
 * src/dpu/src/hash.c includes it but uses nothing from it, so the host compiler
 * can build that file unchanged for the hash golden vectors. */
#pragma once
