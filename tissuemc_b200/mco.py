"""Reader of MCML output files (.mco), as written by tmc_b200_write_mco.

Returns the sections as numpy arrays keyed by MCML's section names (InParm values under "photons",
"dz", "dr", "nz", "nr", "na", "n_above", "n_below", "layers"; RAT under "specular", "rd", "a", "tt";
then "A_l", "A_z", "Rd_r", "Rd_a", "Tt_r", "Tt_a", "A_rz" (nr, nz), "Rd_ra" and "Tt_ra" (nr, na)).
Comments start with '#'; values are whitespace-separated, so the reader does not depend on line
breaks inside a section."""

from __future__ import annotations

from pathlib import Path

import numpy as np

_SECTIONS = ("A_l", "A_z", "Rd_r", "Rd_a", "Tt_r", "Tt_a", "A_rz", "Rd_ra", "Tt_ra")


def _tokens(text: str) -> list[str]:
    out = []
    for line in text.splitlines():
        body = line.split("#", 1)[0]
        out.extend(body.split())
    return out


def read_mco(path: str | Path) -> dict:
    tok = _tokens(Path(path).read_text())
    if not tok or tok[0] != "A1":
        raise ValueError(f"{path}: not an MCML output file (version A1 expected)")
    i = tok.index("InParm") + 1
    out: dict = {"file": tok[i]}
    i += 2  # name, 'A'
    out["photons"] = int(float(tok[i]))
    out["dz"], out["dr"] = float(tok[i + 1]), float(tok[i + 2])
    out["nz"], out["nr"], out["na"] = int(tok[i + 3]), int(tok[i + 4]), int(tok[i + 5])
    nl = int(tok[i + 6])
    out["n_above"] = float(tok[i + 7])
    i += 8
    out["layers"] = np.array([[float(t) for t in tok[i + 5 * l:i + 5 * l + 5]] for l in range(nl)])
    i += 5 * nl
    out["n_below"] = float(tok[i])
    i = tok.index("RAT") + 1
    out["specular"], out["rd"], out["a"], out["tt"] = (float(t) for t in tok[i:i + 4])
    sizes = {"A_l": nl, "A_z": out["nz"], "Rd_r": out["nr"], "Rd_a": out["na"], "Tt_r": out["nr"],
             "Tt_a": out["na"], "A_rz": out["nr"] * out["nz"], "Rd_ra": out["nr"] * out["na"],
             "Tt_ra": out["nr"] * out["na"]}
    for key in _SECTIONS:
        j = tok.index(key, i) + 1
        out[key] = np.array([float(t) for t in tok[j:j + sizes[key]]])
        i = j + sizes[key]
    out["A_rz"] = out["A_rz"].reshape(out["nr"], out["nz"])
    out["Rd_ra"] = out["Rd_ra"].reshape(out["nr"], out["na"])
    out["Tt_ra"] = out["Tt_ra"].reshape(out["nr"], out["na"])
    return out


def bin_measures(nr: int, dr: float, na: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(annulus areas [cm^2], ring solid angles [sr], bin-centre cosines) of MCML's scaling."""
    i = np.arange(nr)
    area = 2.0 * np.pi * (i + 0.5) * dr * dr
    da = np.pi / (2 * na)
    a = (np.arange(na) + 0.5) * da
    return area, 4.0 * np.pi * np.sin(a) * np.sin(0.5 * da), np.cos(a)
