"""Host logic of the waterfall / sweep driver: the reference's bit budgets
(reference lib/BER_example.cc:142-166, lib/Capacity_plot_example.cc:91,150-160),
the BER-crossing interpolation and the CSV table. No device needed."""
import math

from wimax_ldpc_lib_b200 import waterfall as wf


def test_ber_example_budgets():
    # pilot: 46080 bits in whole frames
    assert wf.pilot_frames(576) == 80 and wf.pilot_frames(2304) == 20
    # no pilot error: 3.912 / 1e-8 bits
    assert wf.ber_example_frames(0.0, 2304) == math.floor(3.912 / 1e-8) // 2304 == 169791
    # otherwise 10 * floor(3.912 / BER) bits
    assert wf.ber_example_frames(1e-3, 576) == 10 * 3912 // 576
    assert wf.capacity_frames(2304) == 391200 // 2304 + 1 == 170
    assert wf.capacity_frames(576) == 680


def test_ebno_at_interpolates_log_linear():
    pts = [{"ebno_db": 1.0, "ber": 1e-3}, {"ebno_db": 1.1, "ber": 1e-4}, {"ebno_db": 1.2, "ber": 1e-6}]
    assert abs(wf.ebno_at(pts, 1e-5) - 1.15) < 1e-12
    assert abs(wf.ebno_at(pts, 1e-4) - 1.1) < 1e-12
    assert wf.ebno_at(pts[:2], 1e-5) is None
    # a point without errors after one above the target counts as the crossing
    assert wf.ebno_at([{"ebno_db": 2.0, "ber": 1e-4}, {"ebno_db": 2.1, "ber": 0.0}], 1e-5) == 2.1


def test_csv_rows(tmp_path):
    res = {"codes": [{"rate": "1/2", "z": 96, "decoders": {
        "plain": {"points": [{"ebno_db": 1.0, "frames": 10, "fer": 0.5, "ber": 0.1, "bit_errors": 3,
                              "ber_reference_definition": 0.2, "mean_iterations": 5.0, "info_gbps": 30.0}]},
        "learned": {"points": []}}}]}
    p = tmp_path / "w.csv"
    wf.write_csv(res, str(p))
    lines = p.read_text().splitlines()
    assert lines[0].split(",") == wf.CSV_FIELDS
    assert lines[1] == "1/2,96,plain,1.0,10,0.5,0.1,3,0.2,5.0,30.0" and len(lines) == 2
