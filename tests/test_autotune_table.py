"""The autotuner's table (efdc_xm_tune_lookup), on the CPU.

A table is a text file with one line per measured workload:
``<key> | variant=.. ctas_mv=.. ctas_up=.. iters=.. poly=.. margin=.. tol=.. | ms=..``.
A lookup returns the schedule of the last line whose key equals the one asked
for, skips lines that do not parse or hold values out of range, and reports
a missing key as EFDC_XM_BAD_ARGUMENT, so that the same table always gives
the same schedule.  Lines without the inner tolerance (written before it was
a knob) read as its default, 60.
"""
import efdc_xm as X

KEY = "prec=mixed members=2^8 cells=2^24 asym=0 chan=0"


def line(key, v, mv, up, it, poly, mg, ms=1.0, tol=None):
    t = "" if tol is None else f" tol={tol}"
    return (f"{key} | variant={v} ctas_mv={mv} ctas_up={up} iters={it} poly={poly} "
            f"margin={mg}{t} | ms={ms:.4f}\n")


def test_lookup_takes_last_matching_line(tmp_path):
    t = tmp_path / "tune.txt"
    t.write_text(line(KEY, 0, 0, 0, 4, 10, 0) + line("prec=fp64 members=2^8 cells=2^24 asym=0 chan=0",
                                                     1, 0, 0, 8, 10, 0) +
                 line(KEY, 2, 3, 2, 2, 40, 1, tol=50) +
                 line(KEY + " ", 1, 1, 1, 1, 1, 1))  # another key (trailing blank)
    s = X.tune_lookup(t, KEY)
    assert s == {"kernel_variant": 2, "ctas_matvec": 3, "ctas_update": 2, "graph_iters": 2,
                 "poly_threshold": 40, "inner_margin": 1, "inner_tol": 50}
    old = X.tune_lookup(t, "prec=fp64 members=2^8 cells=2^24 asym=0 chan=0")
    assert old["graph_iters"] == 8 and old["inner_tol"] == 60


def test_lookup_skips_bad_lines_and_missing_keys(tmp_path):
    t = tmp_path / "tune.txt"
    t.write_text(line(KEY, 0, 0, 0, 4, 10, 0) + line(KEY, 7, 0, 0, 4, 10, 0) +  # variant 7
                 f"{KEY} | variant=1 garbage\n" + line(KEY, 1, 0, 0, 99, 10, 0) +  # iters 99
                 line(KEY, 1, 0, 0, 4, 10, 0, tol=90))  # tolerance out of range
    assert X.tune_lookup(t, KEY)["kernel_variant"] == 0
    assert X.tune_lookup(t, "prec=mixed members=2^1 cells=2^10 asym=0 chan=0") is None
    assert X.tune_lookup(tmp_path / "missing.txt", KEY) is None
