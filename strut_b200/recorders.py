"""Strut's transient recorder files from a recorded history.

Restates the recorder loop of Strut's transient driver (transient_nonlinear.mojo:1550-1700 for
the file names, 3225-3500 for the per-step rows, 3621 for the envelope flush) on the history the
device returns (`Analysis.history`: displacements at `Model.record_dofs`, global end forces of
`Model.record_elements`):

* node_displacement        `<output>_node<id>.out`, one row per step: the node's requested dofs
* element_force            `<output>_ele<id>.out`, one row per step: the 2 ndf global end forces
* drift                    `<output>_i<i>_j<j>.out`, one value per step: (u_j - u_i) / dx, dx the
                           coordinate difference along perp_dirn (helpers.mojo:3113-3142)
* section_force / section_deformation
                           `<output>_ele<id>_sec<n>.out`, one row per step: the section's
                           resultants or deformations (StrutSectionRecord gives their order;
                           transient_nonlinear.mojo:1631-1655, 3537-3605)
* envelope_node_displacement / envelope_element_force
                           three rows after the last step: component-wise minima, maxima and
                           absolute maxima, the first step's values as the start
                           (helpers.mojo:3153-3200)

Rows are space-separated values ending in a newline (`_format_values_line`, helpers.mojo:2581-2588),
each value in shortest round-trip decimal form; Strut's comparator reads the numbers, its
tolerances apply to the values.  Recorders that share a file append to it in recorder order,
step by step, as Strut's buffers do.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np


def format_values_line(values) -> str:
    return " ".join(repr(float(v)) for v in values) + "\n"


def recorder_outputs(model, disp: np.ndarray, eforce: np.ndarray, sections=None) -> dict:
    """{file name: text} for the recorders of `model`; disp is steps x len(record_dofs), eforce
    steps x len(record_elements) x (2 ndf), sections steps x model.num_record_sections x width
    (needed only when the model has section recorders)."""
    disp = np.asarray(disp, dtype=np.float64)
    eforce = np.asarray(eforce, dtype=np.float64)
    steps = disp.shape[0] if disp.ndim == 2 else eforce.shape[0]
    order, parts, env = [], {}, {}

    def buf(name):
        if name not in parts:
            order.append(name)
            parts[name] = []
        return parts[name]

    for rec in model.recorder_plan:  # every file exists, in recorder order, even when empty
        buf(rec["file"])
    for k in range(steps):
        for rec in model.recorder_plan:
            t = rec["type"]
            if t in ("node_displacement", "envelope_node_displacement"):
                values = disp[k, rec["disp_cols"]]
            elif t in ("element_force", "envelope_element_force"):
                values = eforce[k, rec["elem_col"], :]
            elif t in ("section_force", "section_deformation"):
                values = np.asarray(sections)[k, rec["sec_col"], :]
            else:  # drift
                values = np.array([(disp[k, rec["j_col"]] - disp[k, rec["i_col"]]) / rec["dx"]])
            if t.startswith("envelope_"):
                e = env.get(rec["file"])
                if e is None:
                    env[rec["file"]] = [values.copy(), values.copy(), np.abs(values)]
                else:
                    e[0] = np.where(values < e[0], values, e[0])
                    e[1] = np.where(values > e[1], values, e[1])
                    e[2] = np.where(np.abs(values) > e[2], np.abs(values), e[2])
            else:
                buf(rec["file"]).append(format_values_line(values))
    for name, (mn, mx, ab) in env.items():
        buf(name).extend([format_values_line(mn), format_values_line(mx), format_values_line(ab)])
    return {name: "".join(parts[name]) for name in order}


def write_outputs(model, disp, eforce, outdir, sections=None) -> list:
    """Writes the recorder files into outdir; returns their paths."""
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    paths = []
    for name, text in recorder_outputs(model, disp, eforce, sections).items():
        p = outdir / name
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_text(text)
        paths.append(p)
    return paths


def read_rows(path) -> np.ndarray:
    """The rows of a recorder file as a 2-D array."""
    rows = [list(map(float, ln.split())) for ln in Path(path).read_text().splitlines() if ln.strip()]
    return np.array(rows, dtype=np.float64)
