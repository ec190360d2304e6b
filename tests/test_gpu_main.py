"""GPU: the command-line driver end to end against the reference's own driver.

bsnn_main and the reference's main_buryn (built unchanged from its sources into
oracle/_ref/main_buryn, `make -C oracle refmain`) run the same JSON configuration into two output
directories.  With the background noise off both runs are deterministic, so:
  * the generated location, weight and stimulus files are byte-identical;
  * the spike recordings have the same rows and labels, identical spikes over the first steps (the
    GEMV summation orders differ, so chaotic divergence eventually separates the rasters) and
    population spike counts within 10 % over the whole run;
  * the voltage files carry the same names and neuron ids, and the step-0 weight recording the same
    (pre, post) pairs with weights within 1e-5 relative.
"""
from __future__ import annotations

import filecmp
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from test_config import small_config

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
MAIN = ROOT / "example-cuda-spiking-nn_b200" / "bsnn_main"
REF_MAIN = ROOT / "oracle" / "_ref" / "main_buryn"


def spike_rows(path):
    """{label: sorted neuron ids} of a spike recording (its first line is the header)."""
    rows = {}
    for line in Path(path).read_text().splitlines()[1:]:
        label, _, ids = line.partition(",")
        rows[int(label)] = sorted(int(x) for x in ids.split())
    return rows


def config(out_dir, form=None):
    c = small_config(out_dir, simulation_steps=10002, group_e_mean_background_excitatory_spikes=0.0,
                     stimulus_input_values=[0.6e-9, 0.45e-9], stimulus_start_clock_steps=[50, 4000],
                     stimulus_end_clock_steps=[3000, 9000],
                     stimulus_selected_input_ids=list(range(0, 100, 3)),
                     stimulus_selected_input_post_group_offsets=[0] * len(range(0, 100, 3)),
                     e_e_plasticity_ltp_A=2e-12, e_e_plasticity_ltp_B=4e-12, e_e_plasticity_ltd_A=1e-12,
                     e_e_plasticity_ltd_B=1e-12, i_e_plasticity_ltp_A=1e-12, i_e_plasticity_ltd_A=1e-12,
                     i_e_plasticity_ltd_B=0.2)
    return c


@pytest.mark.skipif(not (MAIN.exists() and REF_MAIN.exists()), reason="bsnn_main or the reference driver not built")
def test_driver_matches_the_reference_driver(tmp_path):
    cfg_ours = tmp_path / "ours.json"
    cfg_ref = tmp_path / "ref.json"
    cfg_ours.write_text(json.dumps(config(tmp_path / "ours")))
    cfg_ref.write_text(json.dumps(config(tmp_path / "ref")))
    p = subprocess.run([str(MAIN), str(cfg_ours)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    p = subprocess.run([str(REF_MAIN), str(cfg_ref)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    for sub in ("locations", "weights", "stimulus_schedules"):
        for f in sorted((ref / sub).glob("*.txt")):
            if f.name.endswith("_recordings_step0.txt") or "recordings" in f.name:
                continue
            assert filecmp.cmp(ours / sub / f.name, f, shallow=False), f
    # spikes
    n_steps = 10000
    for name, n_pop in (("spikes_e.txt", 100), ("spikes_i.txt", 25)):
        a, b = spike_rows(ours / "recordings" / name), spike_rows(ref / "recordings" / name)
        assert sorted(a) == sorted(b) and len(a) == n_steps, (name, len(a), len(b))
        early = [t for t in sorted(b)[:300]]
        assert all(a[t] == b[t] for t in early), (name, [t for t in early if a[t] != b[t]][:5])
        na, nb = sum(len(v) for v in a.values()), sum(len(v) for v in b.values())
        print(f"{name}: {na} spikes vs reference {nb}")
        assert nb > 50 and abs(na - nb) <= 0.10 * nb, (name, na, nb)
    # voltage files: names and ids
    va = sorted(f.name for f in (ours / "recordings").glob("voltages_step*.txt"))
    vb = sorted(f.name for f in (ref / "recordings").glob("voltages_step*.txt"))
    assert va == vb and len(va) >= n_steps  # one file per ring slot and record (the step-0 record included)
    for name in va[:3]:
        la = (ours / "recordings" / name).read_text().splitlines()
        lb = (ref / "recordings" / name).read_text().splitlines()
        assert [x.split(",")[0] for x in la] == [x.split(",")[0] for x in lb]
    # the step-0 weight recording
    wa = (ours / "weights" / "weights_e_to_e_recordings_step0.txt").read_text().splitlines()
    wb = (ref / "weights" / "weights_e_to_e_recordings_step0.txt").read_text().splitlines()
    assert wa[0] == wb[0] and len(wa) == len(wb)
    ka = np.array([[float(v) for v in x.split(",")] for x in wa[1:]])
    kb = np.array([[float(v) for v in x.split(",")] for x in wb[1:]])
    np.testing.assert_array_equal(ka[:, :2], kb[:, :2])
    np.testing.assert_allclose(ka[:, 2], kb[:, 2], rtol=1e-5, atol=1e-5 * float(np.max(np.abs(kb[:, 2]))))
