"""uv-data tables as CSV files.

The imaging path takes its data as pandas DataFrames with the column names
of SMILI's tables: VisTable (complex visibilities or amplitudes), BSTable
(closure phases) and CATable (log closure amplitudes).  These functions read
and write the reference's CSV files of those tables:

- ``read_vistable`` / ``read_bstable`` / ``read_catable`` follow
  smili/uvdata/uvtable/vistable.py:3461-3480, bstable.py:1224-1243 and
  catable.py:1196-1215: ``pandas.read_csv`` with the caller's keyword
  arguments (floats parsed exactly unless the caller chooses another
  ``float_precision``), then the ``utc`` column (when present) parsed into
  datetimes.
  ``uvunit`` only sets the reference's plotting unit and is accepted and
  ignored here.
- ``to_csv`` follows ``UVTable.to_csv`` (smili/uvdata/uvtable/uvtable.py:
  185-202): no index column, pandas' own float formatting (which the
  reference ends up using as well), so every float64 round-trips exactly.

The ``*_COLUMNS`` lists give the reference's column order for each table,
used to write files that the reference reads back.
"""
from __future__ import annotations

import pandas as pd

VIS_COLUMNS = ["utc", "gsthour", "freq", "stokesid", "ifid", "chid", "ch", "u", "v", "w", "uvdist",
               "subarray", "st1", "st2", "st1name", "st2name", "amp", "phase", "weight", "sigma"]
BS_COLUMNS = ["utc", "gsthour", "freq", "stokesid", "chid", "ifid", "ch",
              "u12", "v12", "w12", "uvdist12", "u23", "v23", "w23", "uvdist23", "u31", "v31", "w31", "uvdist31",
              "uvdistmin", "uvdistmax", "uvdistave", "st1", "st2", "st3", "st1name", "st2name", "st3name",
              "amp", "phase", "sigma"]
CA_COLUMNS = ["utc", "gsthour", "freq", "stokesid", "ifid", "chid", "ch",
              "u1", "v1", "w1", "uvdist1", "u2", "v2", "w2", "uvdist2", "u3", "v3", "w3", "uvdist3",
              "u4", "v4", "w4", "uvdist4", "uvdistmin", "uvdistmax", "uvdistave",
              "st1", "st2", "st3", "st4", "st1name", "st2name", "st3name", "st4name",
              "amp", "sigma", "logamp", "logsigma"]

# columns the imaging path reads from each table
VIS_NEEDS = ["u", "v", "amp", "phase", "sigma"]
BS_NEEDS = ["u12", "v12", "u23", "v23", "u31", "v31", "amp", "phase", "sigma"]
CA_NEEDS = ["u1", "v1", "u2", "v2", "u3", "v3", "u4", "v4", "logamp", "logsigma"]


def _read(filename, **args) -> pd.DataFrame:
    args.setdefault("float_precision", "round_trip")  # exact float64 values (pandas' default parser is not)
    table = pd.read_csv(filename, **args)
    if "utc" in table.columns:
        table["utc"] = pd.to_datetime(table["utc"])
    return table


def read_vistable(filename, uvunit=None, **args) -> pd.DataFrame:
    """A VisTable CSV (complex visibilities; also the amplitude table)."""
    return _read(filename, **args)


def read_bstable(filename, uvunit=None, **args) -> pd.DataFrame:
    """A BSTable CSV (bispectra / closure phases)."""
    return _read(filename, **args)


def read_catable(filename, uvunit=None, **args) -> pd.DataFrame:
    """A CATable CSV (closure amplitudes)."""
    return _read(filename, **args)


def to_csv(table: pd.DataFrame, filename, **args) -> None:
    """Write a table as the reference does: no index column."""
    table.to_csv(filename, index=False, index_label=False, **args)


def missing_columns(table: pd.DataFrame, kind: str) -> list:
    """Columns the imaging path needs that ``table`` lacks (kind: "vis",
    "amp", "bs" or "ca")."""
    need = {"vis": VIS_NEEDS, "amp": ["u", "v", "amp", "sigma"], "bs": BS_NEEDS, "ca": CA_NEEDS}[kind]
    return [c for c in need if c not in table.columns]
