"""Host logic of the autotuner's table (no GPU): the shipped table parses,
and a partial retune (--keys) keeps every other row."""
import os

import qla_b200.tune as tune


def test_shipped_table_parses_and_covers_the_hot_kernels():
    rows = tune._read_table(tune.DEFAULT_OUT)
    for key in ("F3_rtimes_D:cr", "F3_norm2_D:c", "F3_dot_D:cc", "D3_rtimes_D:cr", "F3_batch_program"):
        assert key in rows, key
    for key, (t, s, g) in rows.items():
        assert t in (64, 128, 256) and 2 <= s <= 8 and g > 0, (key, t, s, g)
    assert rows["F3_batch_program"][0] in (64, 128)  # the batch kernel's launch bounds


def test_partial_retune_keeps_other_rows(tmp_path):
    path = os.path.join(tmp_path, "table.txt")
    tune._write_table(path, {"A:c": (256, 2, 6000.0), "B:cc": (128, 3, 7000.0)}, "test device")
    table = tune._read_table(path)
    assert table == {"A:c": (256, 2, 6000.0), "B:cc": (128, 3, 7000.0)}
    table["B:cc"] = (64, 4, 7100.0)  # what tune(keys=["B"]) does with a new best shape
    tune._write_table(path, table, "test device")
    assert tune._read_table(path) == {"A:c": (256, 2, 6000.0), "B:cc": (64, 4, 7100.0)}
