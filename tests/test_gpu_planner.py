"""spj_plan_describe against the plans spj_plan_create builds on the B200:
the algorithm, fan-out and table the description gives are the ones the
executed plan reports, with this device's SM count and shared memory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_r,n_s,kw", [(1 << 20, 1 << 21, {}), ((1 << 22) + 1, 1 << 23, {}),
                                        (1 << 23, 1 << 24, dict(join_alg="smj")),
                                        (1 << 21, 1 << 23, dict(rank_num=4, rank_set=4, skew_mode=1)),
                                        (1 << 22, 1 << 22, dict(radix_bits=12, join_alg="nl"))])
def test_describe_matches_the_executed_plan(spj, n_r, n_s, kw):
    import torch
    props = torch.cuda.get_device_properties(0)
    smem = getattr(props, "shared_memory_per_block_optin", spj.B200_SMEM_PER_BLOCK)
    design = spj.make_design(**kw)
    want = spj.describe(n_r, n_s, design, num_sms=props.multi_processor_count, max_smem_per_block=smem)
    R, S, _ = spj.generate_host(n_r, n_s, 1.0, seed=81)
    plan = spj.Plan(n_r, n_s, design)
    dR = torch.from_numpy(R.view(np.int32)).cuda()
    dS = torch.from_numpy(S.view(np.int32)).cuda()
    out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    plan.execute(dR.data_ptr(), dS.data_ptr(), out.data_ptr(), n.data_ptr())
    torch.cuda.synchronize()
    st = plan.stats()
    plan.close()
    assert spj.ALG[want["join_alg"]] == st["join_alg"]
    if want["join_alg"] != "nphj":
        assert (want["radix_bits"], want["table_slots"]) == (st["radix_bits"], st["table_slots"])
