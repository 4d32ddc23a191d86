"""STAR files (read and write), as RELION writes them.

Replaces cryojax/io/_starfile.py, which goes through the ``starfile``
package (absent here).  A STAR file is a sequence of ``data_<name>``
blocks; a block holds either a ``loop_`` table (``_rlnLabel #k`` column
headers, then one whitespace-separated row per line) or ``_rlnLabel value``
pairs.  Each block becomes a pandas DataFrame keyed by its name (a
key-value block is a one-row frame), as ``starfile.read(always_dict=True)``
returns them.  Column types are inferred per column: integers, then
floats, else strings.
"""

from __future__ import annotations

import pathlib
import shlex

import numpy as np
import pandas as pd


def _check_star_path(filename, mode: str):
    """STAR files are named *.star with no other suffix (the same rule on read and write)."""
    path = pathlib.Path(filename)
    if path.suffixes != [".star"]:
        action = "write" if mode == "w" else "read"
        raise OSError(f"cannot {action} {str(path)!r} as a STAR file: its name must end in '.star' "
                      f"(and carry no other suffix), found {path.suffixes or 'none'}")


def _typed(values: list[str]) -> pd.Series:
    for cast in (int, float):
        try:
            return pd.Series([cast(v) for v in values], dtype=("int64" if cast is int else "float64"))
        except ValueError:
            continue
    return pd.Series(values, dtype=object)


def _split(line: str) -> list[str]:
    return shlex.split(line, posix=True) if ("'" in line or '"' in line) else line.split()


def _finish(name, columns, rows, pairs, out):
    if name is None:
        return
    if columns:
        data = {c: _typed([r[i] for r in rows]) for i, c in enumerate(columns)}
        out[name] = pd.DataFrame(data, columns=columns)
    elif pairs:
        out[name] = pd.DataFrame({k: _typed([v]) for k, v in pairs})
    else:
        out[name] = pd.DataFrame()


def read_starfile(filename) -> dict[str, pd.DataFrame]:
    """Every block of a STAR file as {block name: DataFrame}.  cryojax/io/_starfile.py:12-20."""
    _check_star_path(filename, "r")
    out: dict[str, pd.DataFrame] = {}
    name, columns, rows, pairs, in_loop = None, [], [], [], False
    with open(filename) as f:
        for raw in f:
            line = raw.strip()
            if not line or line.startswith("#"):
                if in_loop and rows and not line:
                    in_loop = False  # a blank line ends the table
                continue
            if line.startswith("data_"):
                _finish(name, columns, rows, pairs, out)
                name, columns, rows, pairs, in_loop = line[5:], [], [], [], False
            elif line == "loop_":
                in_loop, columns, rows = True, [], []
            elif line.startswith("_"):
                parts = line.split(None, 1)
                label = parts[0][1:]
                if in_loop and not rows:
                    columns.append(label)
                else:
                    pairs.append((label, parts[1].strip() if len(parts) > 1 else ""))
            elif in_loop and columns:
                fields = _split(line)
                if len(fields) != len(columns):
                    raise ValueError(f"{filename}: row with {len(fields)} fields in a {len(columns)}-column table "
                                     f"(block data_{name})")
                rows.append(fields)
            else:
                raise ValueError(f"{filename}: cannot parse line {line!r}")
    _finish(name, columns, rows, pairs, out)
    return out


def _format(v) -> str:
    if isinstance(v, (float, np.floating)):
        return "nan" if np.isnan(v) else f"{float(v):.6f}"
    if isinstance(v, (bool, np.bool_)):
        return str(int(v))
    s = str(v)
    return f'"{s}"' if (not s or any(c.isspace() for c in s)) else s


def write_starfile(starfile_data: dict[str, pd.DataFrame], filename, **kwargs):
    """Write {block name: DataFrame} as loop_ tables.  cryojax/io/_starfile.py:23-29."""
    _check_star_path(filename, "w")
    if kwargs.get("overwrite") is False and pathlib.Path(filename).exists():
        raise FileExistsError(str(filename))
    lines = ["# Created by cryojax_b200", ""]
    for name, df in starfile_data.items():
        lines += ["", f"data_{name}", "", "loop_"]
        lines += [f"_{c} #{i + 1}" for i, c in enumerate(df.columns)]
        cols = [df[c].to_numpy() for c in df.columns]
        for r in range(len(df)):
            lines.append("\t".join(_format(col[r]) for col in cols))
        lines.append("")
    with open(filename, "w") as f:
        f.write("\n".join(lines) + "\n")
