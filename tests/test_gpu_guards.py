"""Device loop guards made to fire, on valid input, without faulting.

The reference's Woodcock loop and the rejection loops of its Compton and
Rayleigh samplers are unbounded (MCGPU-PET_kernel.cu:319-342, 1247,
1390-1526).  This library caps them (mcpet_run_opts.max_woodcock_steps and
max_rejections): a photon that reaches a cap is dropped, the trip is counted,
and the run returns MCPET_ERR_DEVICE.  Lowering the caps far below what
physical histories need makes them fire on an ordinary phantom; the run must
report the trips, and the next run with the default caps must be clean and
give the uncapped result again.
"""
import numpy as np
import pytest

import mcpet
import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algorithm", [mcpet.ALGORITHM_EVENTS, mcpet.ALGORITHM_HISTORIES])
@pytest.mark.parametrize("cap", ["woodcock", "rejections"])
def test_lowered_caps_fire_and_are_reported(workdir, algorithm, cap):
    sc = scenes.water_cube_scene(workdir, 5.0e4)
    opts = dict(lane_mode=mcpet.LANES_BALANCED, algorithm=algorithm)
    base = sc.run(mcpet.RunOptions(**opts))
    assert sc.guard_trips() == 0 and base.coincidences > 100
    low = {"max_woodcock_steps": 1} if cap == "woodcock" else {"max_rejections": 1}
    with pytest.raises(mcpet.McpetError) as e:
        sc.run(mcpet.RunOptions(collect_counters=True, **opts, **low))
    assert e.value.status == 7 and "guard" in str(e.value)
    trips = sc.guard_trips()
    assert trips > 100, trips
    again = sc.run(mcpet.RunOptions(**opts))
    assert sc.guard_trips() == 0
    for k in ("trues", "scatter", "spectrum"):
        np.testing.assert_array_equal(getattr(again, k), getattr(base, k), err_msg=k)
    sc.close()


def test_lowered_caps_reported_by_device_entry_point(workdir):
    torch = pytest.importorskip("torch")
    sc = scenes.water_cube_scene(workdir, 5.0e4)
    t = mcpet.device_tallies_for(sc)
    t["counters"] = torch.zeros(10, dtype=torch.int64, device="cuda")
    sc.run_device(t, mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, collect_counters=True, max_woodcock_steps=2))
    torch.cuda.synchronize()
    assert int(t["counters"][9].item()) > 0
    assert sc.guard_trips() == int(t["counters"][9].item())
    sc.run_device(t, mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, collect_counters=True))
    torch.cuda.synchronize()
    assert int(t["counters"][9].item()) == 0 and sc.guard_trips() == 0
    sc.close()
