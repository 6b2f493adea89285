"""The BH solvers' convergence table (rec_mpi.py:85,862-880;
rec_nfp_mpi.py:75,442-458): a DataFrame with the columns iter / err / time,
the initial row at iter -1 with time 0, and the whole table rewritten to
<path_out>/<name> after each row.  Host logic, on the CPU."""
import time
import types

import pandas as pd

from holotomocupy_b200.convtable import log_error, new_table


def _solver(path_out=None):
    s = types.SimpleNamespace(table=new_table(), time_start=time.time())
    if path_out is not None:
        s.path_out = path_out
    return s


def test_rows_and_times():
    s = _solver()
    log_error(s, -1, 2.0, "conv.csv")
    s.time_start -= 1.5            # the first iteration took 1.5 s
    log_error(s, 0, 1.0, "conv.csv")
    log_error(s, 5, 0.25, "conv.csv")
    t = s.table
    assert list(t.columns) == ["iter", "err", "time"]
    assert t["iter"].tolist() == [-1, 0, 5]
    assert t["err"].tolist() == [2.0, 1.0, 0.25]
    assert t["time"].iloc[0] == 0.0
    assert 1.5 <= t["time"].iloc[1] < 10.0
    assert 0.0 <= t["time"].iloc[2] < 1.0     # time_start restarted by the previous row


def test_csv_written_after_each_row(tmp_path):
    out = tmp_path / "run" / "x"
    s = _solver(str(out))
    log_error(s, -1, 3.0, "conv_nfp.csv")
    f = out / "conv_nfp.csv"
    assert f.exists()
    assert f.read_text().splitlines()[0] == "iter,err,time"
    log_error(s, 0, 1.5, "conv_nfp.csv")
    back = pd.read_csv(f)
    assert back["iter"].tolist() == [-1, 0] and back["err"].tolist() == [3.0, 1.5]
    assert "Unnamed: 0" not in back.columns     # no index column


def test_no_csv_without_path_out(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    s = _solver()
    log_error(s, -1, 1.0, "conv.csv")
    assert not list(tmp_path.iterdir())
