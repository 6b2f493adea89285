"""The BH solvers' convergence table (rec_mpi.py:85,862-880;
rec_nfp_mpi.py:75,442-458).

``table`` is a pandas DataFrame with the columns ``iter``, ``err`` and
``time``: one row per logged iteration, ``iter = -1`` for the error before the
first iteration (time 0), otherwise the seconds since the previous row.  When
the solver has a ``path_out`` argument the whole table is rewritten to
``<path_out>/conv.csv`` (``conv_nfp.csv`` for near-field ptychography) after
each row, without the index column.  Each row is also logged at warning
level, as the reference's solvers print it.
"""
import logging
import os
import time

# imported with the package (about a second), not inside the first solver's
# construction, which a caller may be timing
import pandas as pd

logger = logging.getLogger("holotomocupy_b200")

COLUMNS = ["iter", "err", "time"]


def new_table():
    """An empty convergence table."""
    return pd.DataFrame(columns=COLUMNS)


def log_error(solver, i, err, csv_name):
    """Append (i, err, time) to ``solver.table`` and restart
    ``solver.time_start``; write the table to ``<solver.path_out>/csv_name``
    when the solver has a ``path_out``."""
    err = float(err)
    if i == -1:
        elapsed = 0.0
        logger.warning("initial error %.5e", err)
    else:
        elapsed = time.time() - solver.time_start
        logger.warning("iteration %d: %.4f s, error %.5e", i, elapsed, err)
    table = solver.table
    table.loc[len(table)] = [i, err, elapsed]
    solver.time_start = time.time()
    path_out = getattr(solver, "path_out", None)
    if path_out:
        name = os.path.join(str(path_out), csv_name)
        os.makedirs(os.path.dirname(name), exist_ok=True)
        table.to_csv(name, index=False)
