"""Generate / check the binary layout of the FDM C ABI.

``python tests/golden/make_abi_layout.py --reference <dir>`` compiles a probe
against the reference's ``native/include/fullmag_fdm.h`` (found under <dir>)
and writes ``abi_layout.json``: sizeof/offsetof of every struct member and the
value of every enum constant and macro.  ``layout_of(include_dir)`` produces
the same table for any header directory; the tests compare this repository's
include/fullmag_fdm.h against the committed fixture.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "abi_layout.json")

STRUCTS = {
    "fullmag_fdm_grid_desc": ["nx", "ny", "nz", "dx", "dy", "dz"],
    "fullmag_fdm_material_desc": ["saturation_magnetisation", "exchange_stiffness", "damping",
                                  "gyromagnetic_ratio"],
    "fullmag_fdm_plan_desc": [
        "grid", "material", "precision", "integrator", "disable_precession", "enable_exchange",
        "enable_demag", "has_external_field", "external_field_am",
        "demag_kernel_xx_spectrum", "demag_kernel_yy_spectrum", "demag_kernel_zz_spectrum",
        "demag_kernel_xy_spectrum", "demag_kernel_xz_spectrum", "demag_kernel_yz_spectrum",
        "demag_kernel_spectrum_len", "active_mask", "active_mask_len", "region_mask",
        "region_mask_len", "exchange_lut", "exchange_lut_len", "boundary_correction",
        "boundary_phi_floor", "boundary_delta_min", "volume_fraction", "volume_fraction_len",
        "face_link_xp", "face_link_xm", "face_link_yp", "face_link_ym", "face_link_zp",
        "face_link_zm", "delta_xp", "delta_xm", "delta_yp", "delta_ym", "delta_zp", "delta_zm",
        "has_demag_boundary_corr", "demag_corr_target_idx", "demag_corr_source_idx",
        "demag_corr_tensor", "demag_corr_target_count", "demag_corr_stencil_size",
        "initial_magnetization_xyz", "initial_magnetization_len", "adaptive_max_error",
        "adaptive_dt_min", "adaptive_dt_max", "adaptive_headroom"],
    "fullmag_fdm_step_stats": [
        "step", "time_seconds", "dt_seconds", "exchange_energy_joules", "demag_energy_joules",
        "external_energy_joules", "total_energy_joules", "max_effective_field_amplitude",
        "max_demag_field_amplitude", "max_rhs_amplitude", "suggested_next_dt", "wall_time_ns"],
    "fullmag_fdm_device_info": ["name", "compute_capability_major", "compute_capability_minor",
                                "driver_version", "runtime_version"],
    "fullmag_fdm_snapshot_desc": ["cell_count", "component_count", "scalar_bytes", "scalar_type"],
}
CONSTANTS = [
    "FULLMAG_FDM_OK", "FULLMAG_FDM_ERR_INVALID", "FULLMAG_FDM_ERR_CUDA", "FULLMAG_FDM_ERR_INTERNAL",
    "FULLMAG_FDM_MAX_EXCHANGE_REGIONS",
    "FULLMAG_FDM_PRECISION_SINGLE", "FULLMAG_FDM_PRECISION_DOUBLE",
    "FULLMAG_FDM_INTEGRATOR_HEUN", "FULLMAG_FDM_INTEGRATOR_DP45", "FULLMAG_FDM_INTEGRATOR_ABM3",
    "FULLMAG_FDM_INTEGRATOR_RK4", "FULLMAG_FDM_INTEGRATOR_RK23",
    "FULLMAG_FDM_OBSERVABLE_M", "FULLMAG_FDM_OBSERVABLE_H_EX", "FULLMAG_FDM_OBSERVABLE_H_DEMAG",
    "FULLMAG_FDM_OBSERVABLE_H_EXT", "FULLMAG_FDM_OBSERVABLE_H_EFF",
    "FULLMAG_FDM_SNAPSHOT_SCALAR_F32", "FULLMAG_FDM_SNAPSHOT_SCALAR_F64",
    "FULLMAG_FDM_BOUNDARY_NONE", "FULLMAG_FDM_BOUNDARY_VOLUME", "FULLMAG_FDM_BOUNDARY_FULL",
]
ENUM_TYPES = ["fullmag_fdm_precision", "fullmag_fdm_integrator", "fullmag_fdm_observable",
              "fullmag_fdm_snapshot_scalar_type", "fullmag_fdm_boundary_correction"]


def _probe_source() -> str:
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "fullmag_fdm.h"',
             "int main(void) {", '  printf("{");']
    first = True
    for s, fields in STRUCTS.items():
        sep = "" if first else ","
        first = False
        lines.append(f'  printf("{sep}\\"sizeof {s}\\": %zu", sizeof({s}));')
        for f in fields:
            lines.append(f'  printf(",\\"{s}.{f}\\": [%zu, %zu]", offsetof({s}, {f}), sizeof((({s}*)0)->{f}));')
    for e in ENUM_TYPES:
        lines.append(f'  printf(",\\"sizeof {e}\\": %zu", sizeof({e}));')
    for c in CONSTANTS:
        lines.append(f'  printf(",\\"{c}\\": %lld", (long long)({c}));')
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    return "\n".join(lines)


def layout_of(include_dir: str) -> dict:
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "probe.c")
        exe = os.path.join(td, "probe")
        with open(src, "w") as f:
            f.write(_probe_source())
        subprocess.run(["gcc", "-std=c99", "-I", include_dir, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return json.loads(out)


if __name__ == "__main__":
    if len(sys.argv) != 3 or sys.argv[1] != "--reference":
        print(__doc__)
        sys.exit(2)
    layout = layout_of(os.path.join(sys.argv[2], "native", "include"))
    with open(FIXTURE, "w") as f:
        json.dump(layout, f, indent=1, sort_keys=True)
    print(f"wrote {FIXTURE} ({len(layout)} entries)")
