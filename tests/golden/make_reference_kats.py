"""Writes tests/golden/reference_kats.json: the inputs and expected answers of
the reference's own unit tests (tests/unit/*.cu of lsmps-3D), restated as data
so the oracle (CPU) and the CUDA path (GPU) are pinned against the same
known answers.  Each entry cites the reference test lines it restates.

Run:  python tests/golden/make_reference_kats.py
"""

import json
import os


def cube27():
    """27-point cube x, y, z in {-1, 0, 1}, loops iz -> iy -> ix
    (smoke_moment_matrix.cu:18-28 and the other 27-point fixtures)."""
    pts = [(ix, iy, iz) for iz in (-1, 0, 1) for iy in (-1, 0, 1) for ix in (-1, 0, 1)]
    return [p[0] for p in pts], [p[1] for p in pts], [p[2] for p in pts]


def all_pairs(n):
    """All-pairs CSR without self (smoke_moment_matrix.cu:45-56)."""
    offsets, indices = [], []
    for i in range(n):
        offsets.append(len(indices))
        indices.extend(j for j in range(n) if j != i)
    offsets.append(len(indices))
    return offsets, indices


def main():
    x, y, z = cube27()
    off, idx = all_pairs(27)
    kats = {
        "neighbor_search": {
            "source": "tests/unit/smoke_neighbor_search.cu:59-187",
            "fluid": {"x": [0.1, 0.4, 1.1, 1.4, 2.6], "y": [0.1, 0.1, 0.1, 0.7, 2.6], "z": [0.1, 0.1, 0.1, 0.1, 2.6]},
            "walls": {"x": [0.2, 1.2, 2.5], "y": [0.5, 0.1, 2.6], "z": [0.1, 0.1, 2.6]},
            "grid": {"origin": [0.0, 0.0, 0.0], "cell_size": 1.0, "dims": [3, 3, 3]},
            "support_radius": 0.75,
            "max_fluid_neighbors": 4,
            "max_wall_neighbors": 3,
            "expected_fluid_offsets": [0, 1, 3, 5, 6, 6],
            "expected_wall_offsets": [0, 1, 2, 3, 4, 5],
            "expected_fluid_rows": [[1], [0, 2], [1, 3], [2], []],
            "expected_wall_rows": [[0], [0], [1], [1], [2]],
        },
        "surface_detection": {
            "source": "tests/unit/smoke_surface_detection.cu:38-236",
            "fluid": {
                "x": [1.0, 0.4, 1.6, 1.0, 1.0, 1.0, 3.5, 2.5],
                "y": [1.0, 1.0, 1.0, 0.4, 1.6, 1.0, 3.5, 2.5],
                "z": [1.0, 1.0, 1.0, 1.0, 1.0, 1.6, 3.5, 1.0],
            },
            "walls": {
                "x": [1.0, 1.0, 1.0, 0.4, 1.9, 3.1, 2.5, 2.5, 2.5, 2.5],
                "y": [1.0, 1.0, 0.4, 0.4, 2.5, 2.5, 1.9, 3.1, 2.5, 2.5],
                "z": [0.4, 1.6, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.4, 1.6],
            },
            "note": "the reference test leaves wall normals unset (fresh device memory); zero normals are used here",
            "grid": {"origin": [0.0, 0.0, 0.0], "cell_size": 1.0, "dims": [4, 4, 4]},
            "params": {
                "support_radius": 0.75, "near_surface_radius": 0.75, "particle_spacing": 0.6,
                "splash_neighbor_threshold": 2, "number_density_ratio_threshold": 0.75,
                "air_open_ratio_threshold": 0.10, "air_anisotropy_threshold": 0.12,
                "include_wall_neighbors": 1, "wall_normal_independence_threshold": 0.25,
                "virtual_light_cone_cosine": 0.8660254,
            },
            "max_fluid_neighbors": 6,
            "max_wall_neighbors": 4,
            "expected_labels_at": {"0": 1, "1": 2, "6": 3, "7": 0},
            "virtual_light_source": "tests/unit/smoke_surface_detection.cu:238-264",
            "expected_open_count_greater": [1, 0],
            "expected_open_fraction_above": {"6": 0.99},
        },
        "moment_matrix": {
            "source": "tests/unit/smoke_moment_matrix.cu:11-132",
            "fluid": {"x": x, "y": y, "z": z},
            "fluid_offsets": off, "fluid_indices": idx,
            "params": {"support_radius": 4.0, "lsmps_regularization": 1.0e-10, "lsmps_wall_weight_scale": 1.0,
                       "density": 1.0, "gravity": [0.0, 0.0, 0.0]},
            "center": 13,
        },
        "provision": {
            "source": "tests/unit/smoke_provision_explicit_update.cu:39-216",
            "fluid": {"x": x, "y": y, "z": z,
                      "vx": [1.5 + 0.5 * a + 2.0 * a * a for a in x], "vy": [-2.0] * 27,
                      "vz": [0.25 * c for c in z]},
            "surface_type": [3] + [0] * 26,
            "walls": {"x": [-2.0, 2.0], "y": [0.0, 0.0], "z": [0.0, 0.0],
                      "vx": [0.4, -0.1], "vy": [0.2, 0.3], "vz": [-0.5, 0.7]},
            "fluid_offsets": off, "fluid_indices": idx,
            "params": {"support_radius": 4.0, "lsmps_regularization": 1.0e-10, "lsmps_wall_weight_scale": 1.0,
                       "kinematic_viscosity": 0.25, "time_step": 0.2, "gravity": [0.1, -0.2, 0.3]},
            "center": 13,
            "expected_laplacian_x_center": 4.0,
            "tolerance": 2.0e-3,
            "expected_workspace_bytes": (27 + 2) * 3 * 8,
        },
        "ppe_solve": {
            "source": "tests/unit/smoke_ppe_matrix.cu:52-117",
            "row_offsets": [0, 2, 4], "col_indices": [0, 1, 0, 1], "values": [4.0, -1.0, -1.0, 4.0],
            "rhs": [3.0, 3.0], "expected": [1.0, 1.0],
            "negated_rhs": [-3.0, -3.0], "expected_negated_clamped": [0.0, 0.0],
            "tolerance": 2.0e-5,
        },
        "ppe": {
            "source": "tests/unit/smoke_ppe_matrix.cu:119-286",
            "fluid": {"x": x, "y": y, "z": z, "vx": list(x), "vy": [2.0 * b for b in y], "vz": [3.0 * c for c in z]},
            "surface_type": [2] + [0] * 26,
            "fluid_offsets": off, "fluid_indices": idx,
            "params": {"support_radius": 4.0, "lsmps_regularization": 1.0e-10, "time_step": 0.5, "density": 2.0,
                       "gravity": [0.0, 0.0, 0.0]},
            "center": 13,
            "expected_nnz": 27 + 702,
            "expected_divergence_center": 6.0,
            "expected_rhs_center": 12.0,
            "tolerance": 2.0e-3,
            "expected_workspace_bytes": (27 + 1) * 4 + (27 + 702) * (4 + 8) + 27 * 4 * 8,
        },
        "pressure_correction": {
            "source": "tests/unit/smoke_pressure_correction.cu:33-200",
            "fluid": {"x": x, "y": y, "z": z, "vx": [0.5] * 27, "vy": [-0.25] * 27, "vz": [0.75] * 27,
                      "pressure": [20.0 + 2.0 * a - 3.0 * b + 4.0 * c for a, b, c in zip(x, y, z)]},
            "surface_type": [3] + [0] * 26,
            "fluid_offsets": off, "fluid_indices": idx,
            "params": {"support_radius": 4.0, "particle_spacing": 1.0, "lsmps_regularization": 1.0e-10,
                       "time_step": 0.5, "density": 2.0, "ps_displacement_scale": 0.0,
                       "wall_clearance_ratio": 0.0, "velocity_smoothing_strength": 0.0},
            "center": 13,
            "expected_gradient_center": [2.0, -3.0, 4.0],
            "tolerance": 2.0e-3,
            "expected_workspace_bytes": 27 * 9 * 8,
        },
        "workspace_bytes": {
            "source": "src/core/runtime.cu:78-91 and tests/unit/smoke_particle_copy.cu:62-76",
            "spec": {"fluid_capacity": 4, "wall_capacity": 2, "max_fluid_neighbors_per_particle": 2,
                     "max_wall_neighbors_per_particle": 3, "cell_capacity": 8},
            # fluid 4*(7*8+4) + walls 2*9*8 + fluid CSR (5*4 + 8*4) + wall CSR (5*4 + 12*4)
            # + fluid cells (4*2*4 + 8*2*4) + wall cells (2*2*4 + 8*2*4)
            "expected_bytes": 4 * (7 * 8 + 4) + 2 * 9 * 8 + (5 * 4 + 8 * 4) + (5 * 4 + 12 * 4)
            + (4 * 2 * 4 + 8 * 2 * 4) + (2 * 2 * 4 + 8 * 2 * 4),
        },
    }
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(out, "w") as f:
        json.dump(kats, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
