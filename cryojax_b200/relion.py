"""RELION particle stacks: STAR parameters in, batched simulation, MRC stacks out.

Mirrors cryojax/dataset/_particle_data/relion.py (RelionParticleParameterFile,
RelionParticleStackDataset) and particle_simulation.py
(simulate_particle_stack), on this package's STAR and MRC readers
(star.py, mrc.py) and simulator objects.  The unit conversions are the
reference's:

* defocus = (rlnDefocusU + rlnDefocusV) / 2, astigmatism = U - V,
  astigmatism angle = rlnDefocusAngle, phase shift = rlnPhaseShift; Cs,
  amplitude contrast, voltage, pixel size and image size from the
  particle's optics group (relion.py:978-1131);
* pose = EulerAnglePose(-rlnOriginXAngst, -rlnOriginYAngst, -rlnAngleRot,
  -rlnAngleTilt, -rlnAnglePsi) (RELION's origin and angles undo the
  particle's shift and rotation); a psi of -999 (not estimated) reads as 0;
  tilt and psi priors stand in for missing angles; ``inverts_rotation``
  maps (phi, theta, psi) -> (-psi, -theta, -phi) wrapped to [-180, 180);
* the envelope (``loads_envelope``) is FourierGaussian(rlnCtfScalefactor,
  rlnCtfBfactor), or Constant(rlnCtfScalefactor) without a B-factor;
* writing inverts all of the above (relion.py:1384-1570), with
  defocus_offset = the pose's z offset folded into both defoci;
* image names are "<index from 1>@<relative path>", stacks numbered from
  0 with ``n_characters`` digits (relion.py:1620-1710).

Simulation goes through the batched device launch: ``simulate_particle_stack``
hands ``compute_image_fn`` the parameters of up to ``batch_size`` particles
at once (every simulator object here takes a leading batch axis), so one
library call simulates the batch.
"""

from __future__ import annotations

import copy
import pathlib
import re
import warnings
from collections.abc import Callable
from typing import Any

import numpy as np
import pandas as pd

from . import mrc as _mrc
from . import star as _star
from .simulator import (
    AstigmaticCTF,
    BasicImageConfig,
    Constant,
    ContrastTransferTheory,
    EulerAnglePose,
    FourierGaussian,
)

RELION_CTF_OPTICS_ENTRIES = [("rlnSphericalAberration", "float64"), ("rlnAmplitudeContrast", "float64")]
RELION_INSTRUMENT_OPTICS_ENTRIES = [("rlnImageSize", "int64"), ("rlnVoltage", "float64"),
                                    ("rlnImagePixelSize", "float64")]
RELION_CTF_PARTICLE_ENTRIES = [("rlnDefocusU", "float64"), ("rlnDefocusV", "float64"),
                               ("rlnDefocusAngle", "float64"), ("rlnPhaseShift", "float64")]
RELION_POSE_PARTICLE_ENTRIES = [("rlnOriginXAngst", "float64"), ("rlnOriginYAngst", "float64"),
                                ("rlnAngleRot", "float64"), ("rlnAngleTilt", "float64"), ("rlnAnglePsi", "float64")]
RELION_DEFAULT_OPTICS_ENTRIES = [*RELION_INSTRUMENT_OPTICS_ENTRIES, *RELION_CTF_OPTICS_ENTRIES,
                                 ("rlnOpticsGroup", "int64")]
RELION_DEFAULT_PARTICLE_ENTRIES = [*RELION_CTF_PARTICLE_ENTRIES, *RELION_POSE_PARTICLE_ENTRIES,
                                   ("rlnOpticsGroup", "int64")]
RELION_REQUIRED_OPTICS_ENTRIES = RELION_DEFAULT_OPTICS_ENTRIES
RELION_REQUIRED_PARTICLE_ENTRIES = [*RELION_CTF_PARTICLE_ENTRIES, ("rlnOpticsGroup", "int64")]
RELION_SUPPORTED_PARTICLE_ENTRIES = [*RELION_REQUIRED_PARTICLE_ENTRIES, ("rlnCtfBfactor", "float64"),
                                     ("rlnCtfScalefactor", "float64")]


def _empty_frame(entries):
    return pd.DataFrame({c: pd.Series(dtype=d) for c, d in entries})


# ---------------------------------------------------------------------------
# Validation
# ---------------------------------------------------------------------------


_MODES = {"r": "read an existing STAR file", "w": "write a new STAR file"}
_PARAMETER_TYPES = {"image_config": BasicImageConfig, "transfer_theory": ContrastTransferTheory,
                    "pose": EulerAnglePose}


def _checked_mode(mode):
    """The file mode, if it is one of _MODES."""
    if mode not in _MODES:
        options = "; ".join(f"{k!r} to {v}" for k, v in _MODES.items())
        raise ValueError(f"unknown mode {mode!r}: use {options}")
    return mode


def _check_index(owner, index, n_rows):
    """Accept an integer row (negative counts from the end), a slice that starts inside the table, or a
    non-empty one-dimensional integer array; anything else is an IndexError naming the dataset class."""
    name = owner.__name__
    if isinstance(index, (int, np.integer)):
        if not -n_rows <= int(index) < n_rows:
            raise IndexError(f"{name}[{int(index)}]: the STAR file holds {n_rows} particle rows")
        return
    if isinstance(index, slice):
        if index.start is not None and index.start >= n_rows:
            raise IndexError(f"{name}[{index.start}:...]: the slice starts past the {n_rows} particle rows")
        return
    if isinstance(index, np.ndarray):
        if index.ndim != 1 or index.size == 0:
            raise IndexError(f"{name}: an index array must be one-dimensional and non-empty (shape {index.shape})")
        return
    raise IndexError(f"{name} is indexed by an int, a slice or a 1-D integer numpy array, not {type(index).__name__}")


def _check_star_blocks(data):
    """The particles and optics blocks exist and carry every column the reader needs."""
    for block, entries in (("particles", RELION_REQUIRED_PARTICLE_ENTRIES), ("optics", RELION_REQUIRED_OPTICS_ENTRIES)):
        if block not in data:
            raise ValueError(f"the STAR data has no '{block}' block (blocks present: {sorted(data)})")
        missing = sorted({k for k, _ in entries} - set(data[block].columns))
        if missing:
            raise ValueError(f"the STAR '{block}' block lacks the required columns {missing}")


def _check_parameter_types(parameters, require_all=False):
    """Each of pose / transfer_theory / image_config present has the simulator type the writer converts;
    with require_all, all three must be present."""
    if require_all:
        missing = sorted(set(_PARAMETER_TYPES) - set(parameters))
        if missing:
            raise ValueError(f"the parameters lack {missing}: appending needs {sorted(_PARAMETER_TYPES)}")
    for key, cls in _PARAMETER_TYPES.items():
        if key in parameters and not isinstance(parameters[key], cls):
            raise TypeError(f"parameters[{key!r}] should be a {cls.__name__}, got {type(parameters[key]).__name__}")


# ---------------------------------------------------------------------------
# STAR rows -> simulator objects
# ---------------------------------------------------------------------------


def _column(frame, key, default=None):
    if key in frame.columns:
        return frame[key].to_numpy(dtype=float)
    return default


def _optics_group_of(particles: pd.DataFrame, optics: pd.DataFrame) -> pd.Series:
    groups = np.unique(np.asarray(particles["rlnOpticsGroup"]))
    if groups.size > 1:
        raise NotImplementedError("Tried to read multiple particles at once that belong to different optics "
                                  "groups; read one optics group at a time.")
    return optics[optics["rlnOpticsGroup"] == int(groups[0])].iloc[0]


def _invert_rotation(pose: EulerAnglePose) -> EulerAnglePose:
    """relion.py:1198-1208."""
    neg = lambda a: ((-a + 180.0) % 360.0) - 180.0
    o = pose.offset_in_angstroms
    return EulerAnglePose(o[..., 0], o[..., 1], neg(pose.psi_angle), neg(pose.theta_angle), neg(pose.phi_angle),
                          offset_z_in_angstroms=(o[..., 2] if o.shape[-1] == 3 else None))


def _make_parameters(particles: pd.DataFrame, optics: pd.Series, scalar: bool, broadcasts_image_config: bool,
                     loads_envelope: bool, pad_options: dict, inverts_rotation: bool):
    """relion.py:978-1131."""
    n = len(particles)
    pick = (lambda a: a[0]) if scalar else (lambda a: a)
    full = lambda v: np.full(n, float(v))
    du, dv = _column(particles, "rlnDefocusU"), _column(particles, "rlnDefocusV")
    defocus, astig = (du + dv) / 2, du - dv
    angle = _column(particles, "rlnDefocusAngle")
    phase = _column(particles, "rlnPhaseShift")
    cs, ac = full(optics["rlnSphericalAberration"]), full(optics["rlnAmplitudeContrast"])
    envelope = None
    if loads_envelope:
        b = _column(particles, "rlnCtfBfactor")
        amp = _column(particles, "rlnCtfScalefactor")
        if b is None and amp is None:
            warnings.warn("`loads_envelope` was set to True, but no envelope parameters were found. Setting "
                          "envelope as None.")
        elif b is None:
            envelope = Constant(pick(amp))
        else:
            envelope = FourierGaussian(pick(np.ones_like(b) if amp is None else amp), pick(b))
    pixel = float(optics["rlnImagePixelSize"])
    kv = float(optics["rlnVoltage"])
    if broadcasts_image_config and not scalar:
        pixel, kv = full(pixel), full(kv)
    size = int(optics["rlnImageSize"])
    config = BasicImageConfig((size, size), pixel, kv, pad_options=pad_options or None)
    zeros = np.zeros(n)
    ox = _column(particles, "rlnOriginXAngst", zeros)
    oy = _column(particles, "rlnOriginYAngst", zeros)
    rot = _column(particles, "rlnAngleRot", zeros)
    if "rlnAngleTilt" in particles.columns:
        tilt = _column(particles, "rlnAngleTilt")
    else:
        tilt = _column(particles, "rlnAngleTiltPrior", zeros)
    if "rlnAnglePsi" in particles.columns:
        psi = _column(particles, "rlnAnglePsi")
        psi = np.where(psi == -999.0, 0.0, psi)  # RELION's placeholder for an unestimated psi
    else:
        psi = _column(particles, "rlnAnglePsiPrior", zeros)
    pose = EulerAnglePose(pick(-ox), pick(-oy), pick(-rot), pick(-tilt), pick(-psi))
    if inverts_rotation:
        pose = _invert_rotation(pose)
    ctf = AstigmaticCTF(pick(defocus), pick(astig), pick(angle), pick(cs))
    transfer = ContrastTransferTheory(ctf, envelope=envelope, amplitude_contrast_ratio=pick(ac),
                                      phase_shift=pick(phase))
    return config, transfer, pose


# ---------------------------------------------------------------------------
# Simulator objects -> STAR rows
# ---------------------------------------------------------------------------


def _single_value(name, v):
    arr = np.atleast_1d(np.asarray(v, dtype=float))
    if np.unique(arr).size > 1:
        raise ValueError(f"Tried to fill a RELION optics group entry with an array that has multiple unique values "
                         f"('{name}').")
    return arr.ravel()[0]


def _parameters_to_optics_data(parameters, group: int) -> pd.DataFrame:
    """relion.py:1384-1444."""
    if not {"image_config", "transfer_theory"}.issubset(parameters):
        raise ValueError("Tried to add an optics group, but the parameter dictionary did not include "
                         "'image_config' and 'transfer_theory'.")
    cfg, tt = parameters["image_config"], parameters["transfer_theory"]
    if cfg.shape[0] != cfg.shape[1]:
        raise ValueError("When adding optics group to STAR file, found non-square shape in `image_config.shape`.")
    if not isinstance(tt.ctf, AstigmaticCTF):
        raise ValueError("`transfer_theory.ctf` must be type `AstigmaticCTF`.")
    return pd.DataFrame({
        "rlnOpticsGroup": [int(group)], "rlnImageSize": [int(cfg.shape[0])],
        "rlnImagePixelSize": [_single_value("rlnImagePixelSize", cfg.pixel_size)],
        "rlnVoltage": [_single_value("rlnVoltage", cfg.voltage_in_kilovolts)],
        "rlnSphericalAberration": [_single_value("rlnSphericalAberration", tt.ctf.spherical_aberration_in_mm)],
        "rlnAmplitudeContrast": [_single_value("rlnAmplitudeContrast", tt.amplitude_contrast_ratio)],
    })


def _parameters_to_particle_data(parameters, group: int | None = None) -> pd.DataFrame:
    """relion.py:1447-1569."""
    if "pose" not in parameters:
        raise ValueError("Tried to modify parameters in STAR file, but the parameter dictionary did not include "
                         "'pose'.")
    pose = parameters["pose"]
    if not isinstance(pose, EulerAnglePose):
        raise ValueError(f"`pose` must be type `EulerAnglePose`, got {type(pose).__name__}.")
    o = np.atleast_2d(pose.offset_in_angstroms)
    n = o.shape[0]
    cols = {
        "rlnOriginXAngst": -o[:, 0], "rlnOriginYAngst": -o[:, 1],
        "rlnAngleRot": -np.asarray(pose.phi_angle, float), "rlnAngleTilt": -np.asarray(pose.theta_angle, float),
        "rlnAnglePsi": -np.asarray(pose.psi_angle, float),
    }
    if "transfer_theory" in parameters:
        tt = parameters["transfer_theory"]
        if not isinstance(tt.ctf, AstigmaticCTF):
            raise ValueError("`transfer_theory.ctf` must be type `AstigmaticCTF`.")
        dz = 0.0 if pose.offset_z_in_angstroms is None else pose.offset_z_in_angstroms
        df = tt.ctf.defocus_in_angstroms + dz
        cols["rlnDefocusU"] = df + tt.ctf.astigmatism_in_angstroms / 2
        cols["rlnDefocusV"] = df - tt.ctf.astigmatism_in_angstroms / 2
        cols["rlnDefocusAngle"] = tt.ctf.astigmatism_angle
        if isinstance(tt.envelope, FourierGaussian):
            cols["rlnCtfBfactor"] = tt.envelope.b_factor
            cols["rlnCtfScalefactor"] = tt.envelope.amplitude
        elif isinstance(tt.envelope, Constant):
            cols["rlnCtfScalefactor"] = tt.envelope.value
        cols["rlnPhaseShift"] = tt.phase_shift
    out = {}
    for k, v in cols.items():
        v = np.asarray(v, float)
        if v.size == 1:
            out[k] = np.full(n, float(v.ravel()[0]))
        elif v.size == n:
            out[k] = v.ravel()
        else:
            raise ValueError("Found inconsistent number of particles when adding particles to the STAR file.")
    if group is not None:
        out["rlnOpticsGroup"] = np.full(n, int(group), dtype=np.int64)
    frame = pd.DataFrame(out)
    meta = parameters.get("metadata")
    if meta is not None:
        if len(meta) != n:
            raise ValueError("The metadata has a different number of particles from the pose.")
        frame = pd.concat([frame, meta.reset_index(drop=True)], axis="columns", verify_integrity=True)
    return frame


def _next_optics_group(optics: pd.DataFrame) -> int:
    g = np.asarray(optics["rlnOpticsGroup"], dtype=int)
    return (0 if g.size == 0 else int(g[-1])) + 1


# ---------------------------------------------------------------------------
# Parameter file
# ---------------------------------------------------------------------------


class RelionParticleParameterFile:
    """Particle parameters of a RELION STAR file.  relion.py:204-533.

    ``parameter_file[index]`` (int, slice or integer array) returns
    {"image_config", "pose", "transfer_theory", "metadata"} with a leading
    batch axis for a slice or array.
    """

    def __init__(self, path_to_starfile, mode: str = "r", exists_ok: bool = False,
                 selection_filter: dict[str, Callable] | None = None, *, loads_metadata: bool = False,
                 broadcasts_image_config: bool = True, loads_envelope: bool = False,
                 updates_optics_group: bool = False, inverts_rotation: bool = False, pad_options: dict | None = None):
        self._mode = _checked_mode(mode)
        self._pad_options = dict(pad_options or {})
        self.path_to_starfile = pathlib.Path(path_to_starfile)
        self._starfile_data = self._load(selection_filter, exists_ok)
        self.loads_metadata = loads_metadata
        self.broadcasts_image_config = broadcasts_image_config
        self.loads_envelope = loads_envelope
        self.updates_optics_group = updates_optics_group
        self.inverts_rotation = inverts_rotation

    def _load(self, selection_filter, exists_ok):
        p = self.path_to_starfile
        if self._mode == "r":
            if not p.exists():
                raise FileNotFoundError(f"Set `mode = 'r'`, but STAR file {p} does not exist. To write a new STAR "
                                        "file, set `mode = 'w'`.")
            data = _star.read_starfile(p)
            _check_star_blocks(data)
            if selection_filter is not None:
                data["particles"] = _select(data["particles"], selection_filter)
            return {"optics": data["optics"], "particles": data["particles"]}
        if p.exists() and not exists_ok:
            raise FileExistsError(f"Set `mode = 'w'`, but STAR file {p} already exists. Set `exists_ok=True` to "
                                  "start a new one anyway.")
        if selection_filter is not None:
            raise ValueError("A `selection_filter` is only used in `mode = 'r'`.")
        return {"optics": _empty_frame(RELION_DEFAULT_OPTICS_ENTRIES),
                "particles": _empty_frame(RELION_DEFAULT_PARTICLE_ENTRIES)}

    @property
    def mode(self):
        return self._mode

    @property
    def starfile_data(self) -> dict[str, pd.DataFrame]:
        return self._starfile_data

    @starfile_data.setter
    def starfile_data(self, value):
        _check_star_blocks(value)
        self._starfile_data = {"optics": value["optics"], "particles": value["particles"]}

    def copy(self):
        return copy.deepcopy(self)

    def __len__(self):
        return len(self._starfile_data["particles"])

    def __getitem__(self, index):
        particles = self._starfile_data["particles"]
        _check_index(type(self), index, len(particles))
        scalar = isinstance(index, (int, np.integer))
        rows = particles.iloc[[int(index)]] if scalar else particles.iloc[index]
        optics = _optics_group_of(rows, self._starfile_data["optics"])
        config, transfer, pose = _make_parameters(rows, optics, scalar, self.broadcasts_image_config,
                                                  self.loads_envelope, self._pad_options, self.inverts_rotation)
        metadata = None
        if self.loads_metadata:
            known = [k for k, _ in RELION_SUPPORTED_PARTICLE_ENTRIES]
            metadata = rows.drop(columns=[c for c in rows.columns if c in known])
        return {"image_config": config, "pose": pose, "transfer_theory": transfer, "metadata": metadata}

    def __setitem__(self, index, value):
        particles = self._starfile_data["particles"]
        _check_index(type(self), index, len(particles))
        _check_parameter_types(value)
        value = dict(value)
        if "pose" in value and self.inverts_rotation:
            value["pose"] = _invert_rotation(value["pose"])
        optics = self._starfile_data["optics"]
        if self.updates_optics_group:
            group = _next_optics_group(optics)
            update = _parameters_to_particle_data(value, group)
            optics = pd.concat([optics, _parameters_to_optics_data(value, group)], ignore_index=True)
        else:
            update = _parameters_to_particle_data(value)
        for c in update.columns:
            if c not in particles.columns:
                particles[c] = pd.Series(dtype=update[c].dtype)
        idx = np.atleast_1d(np.arange(len(particles))[index])
        particles.loc[particles.index[idx], list(update.columns)] = update.to_numpy()
        self._starfile_data = {"optics": optics, "particles": particles}

    def append(self, value):
        """relion.py:382-419: a new optics group for the appended particles."""
        _check_parameter_types(value, require_all=True)
        value = dict(value)
        if self.inverts_rotation:
            value["pose"] = _invert_rotation(value["pose"])
        optics, particles = self._starfile_data["optics"], self._starfile_data["particles"]
        group = _next_optics_group(optics)
        new_optics = _parameters_to_optics_data(value, group)
        new_particles = _parameters_to_particle_data(value, group)
        optics = pd.concat([optics, new_optics], ignore_index=True) if len(optics) else new_optics
        particles = pd.concat([particles, new_particles], ignore_index=True) if len(particles) else new_particles
        self._starfile_data = {"optics": optics, "particles": particles}

    def save(self, *, overwrite: bool = False, **kwargs):
        p = self.path_to_starfile
        if p.exists() and not overwrite:
            raise FileExistsError(f"Tried saving STAR file, but file {p} already exists; pass overwrite=True.")
        p.parent.mkdir(parents=True, exist_ok=True)
        _star.write_starfile(self._starfile_data, p)


def _select(particles, selection_filter):
    """relion.py:926-975."""
    mask = pd.Series(True, index=particles.index)
    for key, fn in selection_filter.items():
        if key not in particles.columns:
            raise ValueError(f"Included key '{key}' in the `selection_filter`, but it is not in the STAR file.")
        if not callable(fn):
            raise ValueError(f"`selection_filter['{key}']` must be a function returning a boolean mask.")
        m = fn(particles[key])
        if not pd.api.types.is_bool_dtype(np.asarray(m)):
            raise ValueError(f"`selection_filter['{key}']` did not return a boolean mask.")
        mask = mask & np.asarray(m)
    return particles[mask.to_numpy()]


# ---------------------------------------------------------------------------
# Particle stack (images)
# ---------------------------------------------------------------------------


def _format_number(number: int, n_characters: int = 6) -> str:
    return str(int(number)).zfill(n_characters)


def _parse_file_number(filename: str) -> int:
    match = re.search(r"(\d+)\.[^.]+$", filename)
    if match is None:
        raise OSError(f"Could not get the file number from file {filename}.")
    return int(match.group(1))


class RelionParticleStackDataset:
    """Particle images of a RELION project, read from and written to MRC stacks.  relion.py:536-862."""

    def __init__(self, parameter_file: RelionParticleParameterFile, path_to_relion_project, mode: str = "r",
                 mrcfile_settings: dict[str, Any] | None = None, *, loads_parameters: bool = True):
        self._mode = _checked_mode(mode)
        self.parameter_file = parameter_file
        self.path_to_relion_project = pathlib.Path(path_to_relion_project)
        s = dict(mrcfile_settings or {})
        self.mrcfile_settings = dict(prefix=s.get("prefix", ""), output_folder=s.get("output_folder", ""),
                                     delimiter=s.get("delimiter", "_"), n_characters=s.get("n_characters", 6),
                                     overwrite=s.get("overwrite", False), compression=s.get("compression"))
        self.loads_parameters = loads_parameters
        particles = parameter_file.starfile_data["particles"]
        if mode == "w":
            particles["rlnImageName"] = pd.Series([None] * len(particles), index=particles.index, dtype=object)
            self.path_to_relion_project.mkdir(parents=True, exist_ok=True)
        else:
            if "rlnImageName" not in particles.columns:
                raise OSError("Could not find column 'rlnImageName' in the STAR file; set `mode = 'w'` to write "
                              "images.")
            if not self.path_to_relion_project.exists():
                raise FileNotFoundError(f"The RELION project directory {self.path_to_relion_project} does not exist.")

    @property
    def mode(self):
        return self._mode

    def __len__(self):
        return len(self.parameter_file)

    def _load_images(self, rows: pd.DataFrame, shape) -> np.ndarray:
        """relion.py:1211-1261: 'k@path' entries, k counted from 1."""
        names = rows["rlnImageName"].to_numpy()
        images = np.empty((len(names), *shape), dtype=np.float64)
        parsed = []
        for nm in names:
            if not isinstance(nm, str) or "@" not in nm:
                raise ValueError(f"Could not parse 'rlnImageName' entry {nm!r}; expected e.g. '000001@stack.mrcs'.")
            k, f = nm.split("@", 1)
            parsed.append((int(k) - 1, f))
        for fname in dict.fromkeys(f for _, f in parsed):
            data = _mrc.read_array_from_mrc(self.path_to_relion_project / fname, mmap=True, permissive=True)
            stack_shape = data.shape if data.ndim == 2 else data.shape[1:]
            if tuple(stack_shape) != tuple(shape):
                raise ValueError(f"The shape of the MRC with filename {fname} does not match 'rlnImageSize'.")
            for i, (k, f) in enumerate(parsed):
                if f == fname:
                    images[i] = data if data.ndim == 2 else data[k]
        return images

    def __getitem__(self, index):
        pf = self.parameter_file
        particles = pf.starfile_data["particles"]
        _check_index(type(self), index, len(particles))
        scalar = isinstance(index, (int, np.integer))
        rows = particles.iloc[[int(index)]] if scalar else particles.iloc[index]
        if "rlnImageName" not in rows.columns:
            raise OSError(f"No entry 'rlnImageName' for index {index}.")
        size = int(_optics_group_of(rows, pf.starfile_data["optics"])["rlnImageSize"])
        images = self._load_images(rows, (size, size))
        if scalar:
            images = images[0]
        if not self.loads_parameters:
            return {"parameters": None, "images": images}
        return {"parameters": pf[index], "images": images}

    def __setitem__(self, index, value):
        if isinstance(index, np.ndarray):
            raise ValueError("When setting `dataset[index] = ...`, `index` must be an int or a slice.")
        if not isinstance(value, dict) or "images" not in value:
            raise TypeError("`dataset[index] = foo` needs a dict `foo` with key 'images' (and optionally "
                            "'parameters').")
        params = value.get("parameters")
        if params is not None:
            self.parameter_file[index] = params
        idx = np.atleast_1d(np.arange(len(self.parameter_file))[index])
        self.write_images(idx, value["images"], parameters=params)

    def append(self, value):
        if not isinstance(value, dict) or "images" not in value or value.get("parameters") is None:
            raise TypeError("`dataset.append(foo)` needs a dict `foo` with keys 'images' and 'parameters'.")
        start = len(self.parameter_file)
        self.parameter_file.append(value["parameters"])
        self.write_images(np.arange(start, len(self.parameter_file)), value["images"], parameters=value["parameters"])

    def _image_filename(self, index: np.ndarray, particles: pd.DataFrame):
        """relion.py:1638-1690: the stack after the previous particle's gets the next number."""
        last = int(index[0]) - 1
        if len(particles) == 0 or last < 0:
            number = 0
        else:
            prev = particles["rlnImageName"].iloc[last]
            if not isinstance(prev, str):
                raise OSError(f"Could not number the MRC file: the particle at index {last} has no image yet.")
            number = _parse_file_number(prev.split("@", 1)[1]) + 1
        s = self.mrcfile_settings
        stem = _format_number(number, s["n_characters"])
        name = stem if s["prefix"] == "" else s["prefix"] + s["delimiter"] + stem
        rel = str(pathlib.Path(s["output_folder"], name + ".mrcs"))
        names = [_format_number(i + 1, s["n_characters"]) + "@" + rel for i in range(index.size)]
        return self.path_to_relion_project / rel, names

    def write_images(self, index_array, images, parameters=None):
        """relion.py:756-833: one stack file per call, named after the previous one."""
        path, images, pixel = self._prepare_write(index_array, images, parameters)
        self._write_stack(path, images, pixel)

    def _write_stack(self, path, images, pixel):
        path.parent.mkdir(parents=True, exist_ok=True)
        _mrc.write_image_stack_to_mrc(images, pixel, path, overwrite=self.mrcfile_settings["overwrite"],
                                      compression=self.mrcfile_settings["compression"])

    def _prepare_write(self, index_array, images, parameters=None):
        """Validate, name the particles' images in the STAR table and return (path, float32 images, pixel size)."""
        pf = self.parameter_file
        particles, optics = pf.starfile_data["particles"], pf.starfile_data["optics"]
        index_array = np.atleast_1d(np.asarray(index_array, dtype=int))
        if parameters is None:
            g = _optics_group_of(particles.iloc[index_array], optics)
            pixel, dim = float(g["rlnImagePixelSize"]), int(g["rlnImageSize"])
        else:
            pixel = float(np.atleast_1d(parameters["image_config"].pixel_size)[0])
            dim = parameters["image_config"].shape[0]
        images = _to_numpy(images)
        if images.ndim == 2:
            images = images[None]
        if images.ndim != 3 or images.shape[-2:] != (dim, dim):
            raise ValueError(f"Image(s) must be of shape `(n_images, {dim}, {dim})`; got {images.shape}.")
        if images.shape[0] != index_array.size:
            raise ValueError(f"{images.shape[0]} images for {index_array.size} dataset indices.")
        path, names = self._image_filename(index_array, particles)
        if "rlnImageName" not in particles.columns:
            particles["rlnImageName"] = pd.Series([None] * len(particles), index=particles.index, dtype=object)
        particles.loc[particles.index[index_array], "rlnImageName"] = names
        return path, np.asarray(images, dtype=np.float32), pixel


def _to_numpy(images):
    try:
        import torch

        if isinstance(images, torch.Tensor):
            return images.detach().cpu().numpy()
    except ImportError:  # pragma: no cover - torch is a dependency
        pass
    return np.asarray(images)


# ---------------------------------------------------------------------------
# Simulation
# ---------------------------------------------------------------------------


def _index_per_particle(index, args):
    if args is None:
        return None
    if isinstance(args, (tuple, list)):
        return type(args)(_index_per_particle(index, a) for a in args)
    if isinstance(args, dict):
        return {k: _index_per_particle(index, v) for k, v in args.items()}
    return args[index]


def simulate_particle_stack(dataset: RelionParticleStackDataset, compute_image_fn: Callable, constant_args=None,
                            per_particle_args=None, batch_size: int | None = None,
                            images_per_file: int | None = None, **kwargs):
    """Simulate every particle of ``dataset`` and write its image stacks and STAR file.

    particle_simulation.py:22-235.  ``compute_image_fn(parameters,
    constant_args, per_particle_args)`` returns the images of the particles
    in ``parameters``.  With ``batch_size`` it receives up to ``batch_size``
    particles at once (batched simulator objects; one device launch per
    call) and returns [b, H, W]; with ``batch_size=None`` it is called once
    per particle and returns [H, W].  ``images_per_file`` images go to each
    MRC stack (default: all).  ``kwargs`` go to the parameter file's save.
    """
    if dataset.mode == "r":
        raise ValueError("Found that the `dataset` was in reading mode (`mode = 'r'`), but this must be "
                         "instantiated in writing mode (`mode = 'w'`).")
    from concurrent.futures import ThreadPoolExecutor

    n = len(dataset)
    per_file = n if images_per_file is None else int(images_per_file)
    pf = dataset.parameter_file
    # each finished stack is written on a background thread while the next one is simulated;
    # the STAR table's image names are assigned in order on this thread
    with ThreadPoolExecutor(max_workers=1) as writer:
        pending = None
        for start in range(0, n, max(per_file, 1)):
            index = np.arange(start, min(start + per_file, n))
            parameters = pf[index]
            chunks = []
            if batch_size is None:
                for k in index:
                    img = compute_image_fn(pf[int(k)], constant_args, _index_per_particle(k, per_particle_args))
                    chunks.append(_to_numpy(img)[None])
            else:
                for b0 in range(0, index.size, int(batch_size)):
                    sub = index[b0:b0 + int(batch_size)]
                    img = _to_numpy(compute_image_fn(pf[sub], constant_args,
                                                     _index_per_particle(sub, per_particle_args)))
                    chunks.append(img.reshape((-1,) + img.shape[-2:]))
            images = chunks[0] if len(chunks) == 1 else np.concatenate(chunks, axis=0)
            job = dataset._prepare_write(index, images, parameters)
            if pending is not None:
                pending.result()
            pending = writer.submit(dataset._write_stack, *job)
        if pending is not None:
            pending.result()
    pf.save(**kwargs)
