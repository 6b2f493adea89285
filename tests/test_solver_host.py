"""The BH solvers' host logic, on the CPU: the convergence table
(rec_mpi.py:85,862-880; rec_nfp_mpi.py:75,442-458) -- a DataFrame with the
columns iter / err / time, the initial row at iter -1 with time 0, and the
whole table rewritten to <path_out>/<name> after each row; vis_debug's
checkpoints and position-drift log (rec_mpi.py:837-860); and the order of
Rec.BH's loop, with the solver's steps replaced by stand-ins."""
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


def test_vis_debug_writes_checkpoints_and_logs_the_position_drift(caplog):
    """Rec.vis_debug (rec_mpi.py:837-860): every vis_step iterations after
    the first, the state goes to the writer with the normalisation constant,
    and the mean absolute drift of the positions from BH's start is logged
    per distance; without a writer, off-step or at the first iteration
    nothing happens.  Host logic, run on CPU tensors."""
    import numpy as np
    import torch
    from holotomocupy_b200.rec import Rec, position_drift

    calls = []
    writer = types.SimpleNamespace(write_checkpoint=lambda v, i, c: calls.append((i, c)))
    pos0 = torch.zeros(4, 2, 2)
    pos = pos0.clone()
    pos[:, 0, 0] = torch.tensor([1.0, -1.0, 2.0, 0.0])     # distance 0, y: mean |drift| 1
    pos[:, 1, 1] = 0.5                                       # distance 1, x: 0.5
    fake = types.SimpleNamespace(vis_step=2, start_iter=0, norm_const=1.5, pos_init=pos0)
    np.testing.assert_allclose(position_drift(pos, pos0), [[1.0, 0.0], [0.0, 0.5]])
    with caplog.at_level("WARNING", logger="holotomocupy_b200"):
        for i in range(5):
            Rec.vis_debug(fake, {"pos": pos}, i, writer)
        Rec.vis_debug(fake, {"pos": pos}, 6, None)
    assert calls == [(2, 1.5), (4, 1.5)]
    msgs = [r.getMessage() for r in caplog.records]
    assert len(msgs) == 2 and "distance 0: y 1.0000 x 0.0000" in msgs[0] and "distance 1: y 0.0000 x 0.5000" in msgs[0]
    fake.vis_step = -1
    Rec.vis_debug(fake, {"pos": pos}, 4, writer)
    assert len(calls) == 2


def test_bh_loop_order_with_a_writer():
    """Rec.BH's host loop (rec_mpi.py:163-227) with a checkpoint writer: each
    iteration, then its error row, then vis_debug, which checkpoints every
    vis_step iterations after the first; a writer turns mode="graph" into the
    host loop.  The solver's steps are stand-ins; this is the loop's order."""
    import torch
    from holotomocupy_b200.rec import Rec

    calls = []
    fake = types.SimpleNamespace(niter=5, start_iter=0, err_step=-1, vis_step=2, graphable=True, norm_const=2.0,
                                 vars={"pos": torch.zeros(3, 2, 2)}, pos_init=torch.zeros(3, 2, 2))
    fake.bh_setup = lambda: calls.append("setup")
    fake.bh_iteration = lambda i, sync=True: (calls.append(("it", i)), (0.1 * i, 0.2 * i))[1]
    fake.error_debug = lambda v, i: calls.append(("err", i))
    fake.bh_finish = lambda: (calls.append("finish"), fake.vars)[1]
    fake.vis_debug = types.MethodType(Rec.vis_debug, fake)
    writer = types.SimpleNamespace(write_checkpoint=lambda v, i, c: calls.append(("ck", i, c)))
    record = []
    Rec.BH(fake, writer=writer, record=record, mode="graph")
    assert calls == ["setup", ("it", 0), ("err", 0), ("it", 1), ("err", 1), ("it", 2), ("err", 2), ("ck", 2, 2.0),
                     ("it", 3), ("err", 3), ("it", 4), ("err", 4), ("ck", 4, 2.0), "finish"]
    assert [r[0] for r in record] == [0, 1, 2, 3, 4]


def test_bh_graph_mode_of_a_real_object_runs_the_host_loop():
    """mode="graph" on an iteration that cannot be recorded (a real-valued
    object: graphable False) runs the host loop, with the host step sizes."""
    from holotomocupy_b200.rec import Rec

    calls = []
    fake = types.SimpleNamespace(niter=3, start_iter=0, err_step=-1, vis_step=-1, graphable=False, vars={})
    fake.bh_setup = lambda: calls.append("setup")
    fake.bh_iteration = lambda i, sync=True: (calls.append(("it", i, sync)), (1.0, 0.0))[1]
    fake.error_debug = lambda v, i: None
    fake.bh_finish = lambda: (calls.append("finish"), fake.vars)[1]
    Rec.BH(fake, mode="graph")
    assert calls == ["setup", ("it", 0, True), ("it", 1, True), ("it", 2, True), "finish"]
