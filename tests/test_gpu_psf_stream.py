"""PSF records streamed in chunks (mcpet_run_psf_stream): same records (as a
set), sinograms and totals as one run with an unbounded PSF buffer, in both
PSF modes; small chunks exercise the replay of ranges that overflow."""
import numpy as np
import pytest

import mcpet
import scenes

pytestmark = pytest.mark.gpu


def _as_set(rec):
    return np.sort(np.ascontiguousarray(rec).view(np.dtype((np.void, rec.dtype.itemsize))).ravel())


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("chunk", [64, 4096])
def test_stream_equals_unbounded_run(tmp_path, mode, chunk):
    sc = scenes.small_head_scene(str(tmp_path), total_bq=2.0e5, tally_psf_sinogram=mode, psf_size=4_000_000)
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=8)
    full = sc.run(opts)
    assert full.psf_count > 4 * chunk and full.psf_count < 4_000_000
    got = []
    st = sc.run_psf_stream(chunk, opts, sink=lambda r: got.append(r.copy()))
    assert all(len(g) <= chunk for g in got)
    rec = np.concatenate(got)
    assert st.psf_count == full.psf_count == len(rec)
    np.testing.assert_array_equal(_as_set(rec), _as_set(full.psf))
    assert st.total_histories == full.total_histories
    if mode == 0:
        np.testing.assert_array_equal(st.trues, full.trues)
        np.testing.assert_array_equal(st.scatter, full.scatter)
        np.testing.assert_array_equal(st.spectrum, full.spectrum)
        assert st.detected == full.detected
    sc.close()


def test_stream_sink_can_stop(tmp_path):
    sc = scenes.small_head_scene(str(tmp_path), total_bq=1.0e5, tally_psf_sinogram=1, psf_size=1_000_000)
    with pytest.raises(mcpet.McpetError):
        sc.run_psf_stream(256, mcpet.RunOptions(), sink=lambda r: False)
    sc.close()
