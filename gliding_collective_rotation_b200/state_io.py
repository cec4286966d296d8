"""State files in the reference's ``.dat`` format, and resuming from them.

``write_state`` writes what ``output_methods.save_state`` writes for a chain
population (output_methods.py:420-466), byte for byte: the file
``<prefix>_<pop>_<filenumber, zero-padded>.dat`` (or ``<prefix>_<pop>.dat``
when only the most recent state is kept) with the header
``# filenumber F stepnum S t T class <class>`` and one row per bead,
``chain_id inherited_label x y [z] phi [theta] where_active`` -- the
tangents stored as angles (``Chain_Collection.tangents_to_orientations``,
populations.py:559-562).

``read_state`` reads such a file as ``analysis.recall`` does
(analysis.py:23-107), by column name, in 2D and 3D (the reference's reader
takes ``where_active`` from column 5, which in 3D is ``phi``, and misspells
an attribute on its 3D path; here every column is found by its header
name).  ``spec_from_state`` turns a state into a ``SystemSpec`` so a run
resumes from it on the GPU; ``save_batch`` writes every system of a
``Batch``.

Positions and angles are written with 9 significant digits (``%.8e``), as
the reference writes them: a resumed run starts within ~1e-8 relative of
where the saved one was.
"""
from __future__ import annotations

import copy
import os

import numpy as np

DEFAULT_CLASS = "populations.Equal_Size_Chain_Collection"


def zero_padded(number, n_digits):
    """output_methods.zero_padded_string (output_methods.py:343-349)."""
    return ("0" * n_digits)[:-len(str(number))] + str(number)


def state_filename(prefix, filenumber, pop_name="beads", n_digits=8, most_recent_only=False):
    name = f"{prefix}_{pop_name}"
    if not most_recent_only:
        name += "_" + zero_padded(filenumber, n_digits)
    return name + ".dat"


def tangents_to_orientations(tangent):
    """phi (2D) or (phi, theta) (3D) of each tangent."""
    tangent = np.asarray(tangent, dtype=np.float64)
    phi = np.arctan2(tangent[:, 1], tangent[:, 0])
    if tangent.shape[1] == 2:
        return phi[:, None]
    return np.column_stack((phi, np.arccos(tangent[:, 2])))


def orientations_to_tangents(orient):
    orient = np.asarray(orient, dtype=np.float64)
    if orient.shape[1] == 1:
        return np.column_stack((np.cos(orient[:, 0]), np.sin(orient[:, 0])))
    st = np.sin(orient[:, 1])
    return np.column_stack((st * np.cos(orient[:, 0]), st * np.sin(orient[:, 0]), np.cos(orient[:, 1])))


def write_state(prefix, filenumber, stepnum, t, pos, tangent, chain_id, inherited_label=None, where_active=None,
                pop_name="beads", n_digits=8, most_recent_only=False, class_name=DEFAULT_CLASS):
    """Write one chain population's state; returns the file name."""
    pos = np.asarray(pos, dtype=np.float64)
    dim = pos.shape[1]
    chain_id = np.asarray(chain_id)
    inherited_label = chain_id if inherited_label is None else np.asarray(inherited_label)
    where_active = np.zeros(len(pos), dtype=np.int64) if where_active is None else np.asarray(where_active)
    orient = tangents_to_orientations(tangent)
    head = f"filenumber {filenumber} stepnum {stepnum} t {t:.5f} class {class_name}\n"
    fn = state_filename(prefix, filenumber, pop_name, n_digits, most_recent_only)
    if dim == 2:
        cols = (chain_id, inherited_label, pos[:, 0], pos[:, 1], orient[:, 0], where_active)
        fmt = ["%d", "%d", "%.8e", "%.8e", "%.8e", "%d"]
        names = "chain_id inherited_label x y phi where_active inherited_label"
    else:
        cols = (chain_id, inherited_label, pos[:, 0], pos[:, 1], pos[:, 2], orient[:, 0], orient[:, 1], where_active)
        fmt = ["%d", "%d", "%.8e", "%.8e", "%.8e", "%.8e", "%.8e", "%d"]
        names = "chain_id inherited_label x y z phi theta where_active inherited_label"
    np.savetxt(fn, np.column_stack(cols), fmt=fmt, header=head + names)
    return fn


def read_state(filename):
    """A state file as a dict: pos, tangent, orientations, chain_id,
    inherited_label, where_active, stepnum, t, filenumber, class_name."""
    with open(filename) as fh:
        lines = fh.readlines()
    first = lines[0].lstrip("#").split()
    names = lines[1].lstrip("#").split()
    data = np.loadtxt(lines[2:], ndmin=2)
    col = {}
    for i, nm in enumerate(names):
        col.setdefault(nm, i)  # the reference lists inherited_label twice
    out = {"stepnum": int(first[first.index("stepnum") + 1]), "t": float(first[first.index("t") + 1]),
           "filenumber": int(first[first.index("filenumber") + 1]),
           "class_name": first[first.index("class") + 1] if "class" in first else None}
    out["pos"] = np.column_stack([data[:, col[k]] for k in ("x", "y", "z") if k in col])
    orient = np.column_stack([data[:, col[k]] for k in ("phi", "theta") if k in col])
    out["orientations"] = orient
    out["tangent"] = orientations_to_tangents(orient)
    for k in ("chain_id", "inherited_label", "where_active"):
        if k in col:
            out[k] = data[:, col[k]].astype(np.int64)
    return out


def spec_from_state(state, template):
    """A ``SystemSpec`` with ``template``'s parameters and the saved beads;
    the step counter (the Philox key) continues from the saved step."""
    spec = copy.deepcopy(template)
    chain = np.asarray(state["chain_id"])
    if len(chain) != template.n or np.any(np.diff(chain) < 0):
        raise ValueError("the state does not hold the template's chains")
    spec.pos = np.mod(np.asarray(state["pos"], dtype=np.float64), template.params.L)
    spec.tangent = np.asarray(state["tangent"], dtype=np.float64)
    spec.chain_id = chain
    spec.params.step = int(state["stepnum"])
    return spec


def save_batch(batch, prefix, filenumber, t=None, n_digits=8):
    """Write every system of a ``Batch`` (``<prefix><i>_beads_<n>.dat``);
    returns the file names."""
    names = []
    for i, (st, sp) in enumerate(zip(batch.states, batch.statuses())):
        pos = st.pos.cpu().numpy()
        tan = st.tangent.double().cpu().numpy()
        chain = st.chain_id.cpu().numpy()
        time = sp["step"] * batch.specs[i].dt if t is None else t
        names.append(write_state(f"{prefix}{i}", filenumber, sp["step"], time, pos, tan, chain, n_digits=n_digits))
    return names


def save_populations(batch, members, pop_names, prefix, filenumber, stepnum, t, n_digits=8):
    """Write the populations of one box (systems ``members`` of a ``Batch``,
    coupled with ``Batch.couple``) the way ``output_methods.save_state``
    writes a list of populations (output_methods.py:420-466): one file per
    population, ``<prefix>_<pop name>_<n>.dat``, the same file number, step
    and time in every header; returns the file names."""
    names = []
    for i, name in zip(members, pop_names):
        st = batch.states[i]
        names.append(write_state(prefix, filenumber, stepnum, t, st.pos.cpu().numpy(),
                                 st.tangent.double().cpu().numpy(), st.chain_id.cpu().numpy(), pop_name=name,
                                 n_digits=n_digits))
    return names


def latest_state(prefix, pop_name="beads"):
    """The most recent file of a run (highest file number)."""
    d = os.path.dirname(prefix) or "."
    base = os.path.basename(prefix) + f"_{pop_name}"
    files = sorted(f for f in os.listdir(d) if f.startswith(base) and f.endswith(".dat"))
    return os.path.join(d, files[-1]) if files else None
