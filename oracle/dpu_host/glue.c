/* glue.c -- the runner's view of one reference kernel's __host variables: its
 * argument struct set field by field from the runner's integer list (the struct
 * itself comes from the reference's include/argument.h), and its results read
 * back as integers. Built once per kernel with one of -DGLUE_COUNT,
 * -DGLUE_PACKET, -DGLUE_BGCOUNT, -DGLUE_BGALIGN, -DGLUE_BUILD, -DGLUE_PROBE, -DGLUE_NL,
 * -DGLUE_LP, -DGLUE_SMP, -DGLUE_SMJ, -DGLUE_NBUILD, -DGLUE_NPROBE or
 * -DGLUE_FINISH. Test infrastructure of the oracle only. */
#include <stdbool.h>
#include <stdint.h>

#include "dpu_host.h"
#include "argument.h"

extern dpu_results_t dpu_results;

static int errors_out(int64_t *o) {
    o[0] = dpu_results.ERROR_TYPE_0;
    o[1] = dpu_results.ERROR_TYPE_1;
    o[2] = dpu_results.ERROR_TYPE_2;
    o[3] = dpu_results.ERROR_TYPE_3;
    return 4;
}

#if defined(GLUE_COUNT)
/* src/dpu/src/join/glb_partition_count.c and glb_chipwise_partition_count.c */
extern glb_partition_count_arg param_glb_partition_count;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 12) return -1;
    glb_partition_count_arg *p = &param_glb_partition_count;
    p->input_type = (int32_t)a[0];
    p->partition_type = (int32_t)a[1];
    p->input_offset = (int32_t)a[2];
    p->elem_num = (int32_t)a[3];
    p->partition_info_start_byte = (int32_t)a[4];
    p->histogram_start_byte = (int32_t)a[5];
    p->partition_num = (int32_t)a[6];
    p->bankgroup = (int32_t)a[7];
    p->num_rankgroup = (int32_t)a[8];
    p->num_rank_in_rankgroup = (int32_t)a[9];
    p->join_type = (int32_t)a[10];
    p->hist_interval = (int32_t)a[11];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#elif defined(GLUE_PACKET)
/* src/dpu/src/join/glb_partition_packet.c and glb_chipwise_partition_packet.c */
extern glb_partition_packet_arg param_glb_partition_packet;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 18) return -1;
    glb_partition_packet_arg *p = &param_glb_partition_packet;
    p->dpu_id = (int32_t)a[0];
    p->rank_id = (int32_t)a[1];
    p->input_type = (int32_t)a[2];
    p->partition_type = (int32_t)a[3];
    p->input_offset1 = (int32_t)a[4];
    p->input_offset2 = (int32_t)a[5];
    p->elem_num = (int32_t)a[6];
    p->histogram_start_byte = (int32_t)a[7];
    p->packet_histogram_start_byte = (int32_t)a[8];
    p->partition_num = (int32_t)a[9];
    p->result_offset = (int32_t)a[10];
    p->packet_size = (int32_t)a[11];
    p->partition_start = (int32_t)a[12];
    p->bankgroup = (int32_t)a[13];
    p->num_rankgroup = (int32_t)a[14];
    p->num_rank_in_rankgroup = (int32_t)a[15];
    p->join_type = (int32_t)a[16];
    p->hist_interval = (int32_t)a[17];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#elif defined(GLUE_BGCOUNT)
/* src/dpu/src/join/bg_broadcast_count.c */
extern bg_broadcast_count_arg param_bg_broadcast_count;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 8) return -1;
    bg_broadcast_count_arg *p = &param_bg_broadcast_count;
    p->input_offset = (int32_t)a[0];
    p->elem_num = (int32_t)a[1];
    p->partition_info_start_byte = (int32_t)a[2];
    p->histogram_start_byte = (int32_t)a[3];
    p->partition_num = (int32_t)a[4];
    p->bankgroup = (int32_t)a[5];
    p->rankgroup = (int32_t)a[6];
    p->padding = (int32_t)a[7];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#elif defined(GLUE_BGALIGN)
/* src/dpu/src/join/bg_broadcast_align.c */
extern bg_broadcast_align_arg param_bg_broadcast_align;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 10) return -1;
    bg_broadcast_align_arg *p = &param_bg_broadcast_align;
    p->elem_num = (uint32_t)a[0];
    p->partition_num = (uint32_t)a[1];
    p->tid_offset = (uint32_t)a[2];
    p->payload_offset = (uint32_t)a[3];
    p->result_offset = (uint32_t)a[4];
    p->global_histogram_start_byte = (uint32_t)a[5];
    p->aggr_histogram_start_byte = (uint32_t)a[6];
    p->bankgroup = (int32_t)a[7];
    p->rankgroup = (int32_t)a[8];
    p->padding = (int32_t)a[9];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#elif defined(GLUE_BUILD)
/* src/dpu/src/join/a2a_srj_build.c */
extern hash_phj_build_arg param_phj_build_hash_table;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 7) return -1;
    hash_phj_build_arg *p = &param_phj_build_hash_table;
    p->parted_R_offset = (uint32_t)a[0];
    p->parted_Tid_R_offset = (uint32_t)a[1];
    p->HT_offset = (uint32_t)a[2];
    p->parted_R_info_offset = (uint32_t)a[3];
    p->partition_num = (uint32_t)a[4];
    p->R_num = (uint32_t)a[5];
    p->compressed_key = (uint32_t)a[6];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#elif defined(GLUE_PROBE)
/* src/dpu/src/join/a2a_srj_probe_inner_mt.c */
extern hash_phj_probe_arg param_phj_probe_hash_table_inner;
extern hash_phj_probe_return_arg param_hash_phj_probe_return;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 11) return -1;
    hash_phj_probe_arg *p = &param_phj_probe_hash_table_inner;
    p->parted_S_offset = (int32_t)a[0];
    p->parted_Tid_S_offset = (int32_t)a[1];
    p->HT_offset = (int32_t)a[2];
    p->parted_S_info_offset = (int32_t)a[3];
    p->Result_offset = (int32_t)a[4];
    p->partition_num = (int32_t)a[5];
    p->S_num = (int32_t)a[6];
    p->rank_id = (int32_t)a[7];
    p->dpu_id = (int32_t)a[8];
    p->key_table_type = (int32_t)a[9];
    p->probe_type = (int32_t)a[10];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) {
    if (cap < 6) return 0;
    errors_out(o);
    o[4] = param_hash_phj_probe_return.result_size;
    o[5] = param_hash_phj_probe_return.miss_count;
    return 6;
}

#elif defined(GLUE_NL)
/* src/dpu/src/join/nested_loop_join.c */
extern nested_loop_join_arg param_nested_loop_join;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 6) return -1;
    nested_loop_join_arg *p = &param_nested_loop_join;
    p->R_packet_start_byte = (int32_t)a[0];
    p->S_packet_start_byte = (int32_t)a[1];
    p->R_num_packets = (int32_t)a[2];
    p->S_num_packets = (int32_t)a[3];
    p->packet_size = (int32_t)a[4];
    p->result_start_byte = (int32_t)a[5];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#elif defined(GLUE_LP)
/* src/dpu/src/join/a2a_packetwise_srj_local_partition.c */
extern packetwise_hash_local_partitioning_arg param_packetwise_local_hash_partitioning;
extern packetwise_hash_local_partitioning_return_arg param_packetwise_local_hash_partitioning_return;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 12) return -1;
    packetwise_hash_local_partitioning_arg *p = &param_packetwise_local_hash_partitioning;
    p->packet_start_byte = (int32_t)a[0];
    p->generated_local_tid_start_byte = (int32_t)a[1];
    p->partitioned_result_start_byte = (int32_t)a[2];
    p->result_partition_info_start_byte = (int32_t)a[3];
    p->do_calculate_partition_num = (int32_t)a[4];
    p->shift_val = (int32_t)a[5];
    p->total_rank = (int32_t)a[6];
    p->num_packets = (int32_t)a[7];
    p->tuple_size = (int32_t)a[8];
    p->packet_size = (int32_t)a[9];
    p->rank_id = (int32_t)a[10];
    p->dpu_id = (int32_t)a[11];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) {
    if (cap < 6) return 0;
    errors_out(o);
    o[4] = param_packetwise_local_hash_partitioning_return.elem_num;
    o[5] = param_packetwise_local_hash_partitioning_return.partition_num;
    return 6;
}

#elif defined(GLUE_SMP)
/* src/dpu/src/join/mpsm_join_local_partition.c */
extern sort_merge_partitioning_arg param_sort_merge_partitioning;
extern sort_merge_probe_return_arg param_sort_merge_probe_return;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 8) return -1;
    sort_merge_partitioning_arg *p = &param_sort_merge_partitioning;
    p->elem_range = (int32_t)a[0];
    p->num_packets = (int32_t)a[1];
    p->packet_size = (int32_t)a[2];
    p->hist_interval = (int32_t)a[3];
    p->r_packet_start_byte = (int32_t)a[4];
    p->r_sorted_start_byte = (int32_t)a[5];
    p->histogram_addr_start_byte = (int32_t)a[6];
    p->data_skewness = (int32_t)a[7];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) {
    if (cap < 5) return 0;
    errors_out(o);
    o[4] = param_sort_merge_probe_return.result_size;
    return 5;
}

#elif defined(GLUE_SMJ)
/* src/dpu/src/join/mpsm_join_sort_probe.c */
extern sort_merge_sort_probe_arg param_sort_merge_sort_probe;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 9) return -1;
    sort_merge_sort_probe_arg *p = &param_sort_merge_sort_probe;
    p->elem_range = (int32_t)a[0];
    p->hist_interval = (int32_t)a[1];
    p->r_sorted_start_byte = (int32_t)a[2];
    p->s_sorted_start_byte = (int32_t)a[3];
    p->r_histogram_start_byte = (int32_t)a[4];
    p->s_histogram_start_byte = (int32_t)a[5];
    p->result_probe_start_byte = (int32_t)a[6];
    p->r_total_bytes = (int32_t)a[7];
    p->s_total_bytes = (int32_t)a[8];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#elif defined(GLUE_NBUILD)
/* src/dpu/src/join/packetwise_no_partitioned_hash_join_build.c */
extern packetwise_nphj_build_arg param_packetwise_nphj_build;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 4) return -1;
    packetwise_nphj_build_arg *p = &param_packetwise_nphj_build;
    p->R_packet_start_byte = (int32_t)a[0];
    p->num_input_bytes = (int32_t)a[1];
    p->hash_table_start_byte = (int32_t)a[2];
    p->hash_table_byte_size = (int32_t)a[3];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#elif defined(GLUE_NPROBE)
/* src/dpu/src/join/packetwise_no_partitioned_hash_join_probe.c */
extern packetwise_nphj_probe_arg param_packetwise_nphj_probe;
extern packetwise_nphj_probe_return_arg param_packetwise_nphj_probe_return;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 5) return -1;
    packetwise_nphj_probe_arg *p = &param_packetwise_nphj_probe;
    p->S_packet_start_byte = (int32_t)a[0];
    p->num_input_bytes = (int32_t)a[1];
    p->hash_table_start_byte = (int32_t)a[2];
    p->hash_table_byte_size = (int32_t)a[3];
    p->result_start_byte = (int32_t)a[4];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) {
    if (cap < 6) return 0;
    errors_out(o);
    o[4] = param_packetwise_nphj_probe_return.result_size;
    o[5] = param_packetwise_nphj_probe_return.miss_count;
    return 6;
}

#elif defined(GLUE_FINISH)
/* src/dpu/src/join/finish_join.c */
extern finish_join_arg param_finish_join;

int dpu_host_set_args(const int64_t *a, int n) {
    if (n != 4) return -1;
    finish_join_arg *p = &param_finish_join;
    p->join_result_start_byte = (int32_t)a[0];
    p->max_bytes = (int32_t)a[1];
    p->effective_bytes = (int32_t)a[2];
    p->dummy = (int32_t)a[3];
    return 0;
}

int dpu_host_get_results(int64_t *o, int cap) { return cap < 4 ? 0 : errors_out(o); }

#else
#error "define GLUE_COUNT, GLUE_PACKET, GLUE_BGCOUNT, GLUE_BGALIGN, GLUE_FINISH, GLUE_BUILD, GLUE_PROBE, GLUE_NL, GLUE_LP, GLUE_SMP, GLUE_SMJ, GLUE_NBUILD or GLUE_NPROBE"
#endif
