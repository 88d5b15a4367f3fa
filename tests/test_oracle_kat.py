"""The CPU oracle is pinned to the reference's own known-answer tests.

oracle/oracle_kat.cpp restates each #[test] of the reference that covers the render path
(minkowski.rs:615-691, mesh4d.rs:1095-1322, star.rs:329-428, bloom.rs:131-151,
renderer.rs:1140-1211) with the reference's tolerances; this runs it.
"""
import os
import subprocess

from conftest import ROOT

EXPECTED = [
    "cross4_orthogonality", "tetrad_orthonormality_and_null_rays", "relativistic_aberration_formula",
    "worldtube_decided_at_follows_steps", "ray_simplex4d_intersection", "emergent_length_contraction_in_worldtube",
    "thomas_precession_one_orbit", "born_rigid_front_back_proper_time_offset",
    "white_point_is_white_and_doppler_shifts_color", "past_cone_event_is_null_and_in_the_past",
    "star_flux_is_conserved_across_subpixel_positions",
    "polyline_star_is_found_by_segment_and_ends_at_its_last_event", "star_behind_an_occluder_is_hidden",
    "approaching_star_is_blueshifted_and_brighter", "bloom_conserves_energy_and_spreads_a_point",
    "flat_image_is_unchanged", "analytic_decision_age_is_time_ago_plus_distance",
    "analytic_decision_age_on_past_cone_is_round_trip", "haze_covers_every_undecided_cone", "gamma_lut_and_pack",
    "config1_scene_shape",
]


def test_oracle_matches_reference_known_answers():
    exe = os.path.join(ROOT, "oracle", "oracle_kat")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    passed = {line.split()[1] for line in r.stdout.splitlines() if line.startswith("PASS ")}
    assert r.returncode == 0, r.stdout
    assert set(EXPECTED) <= passed, r.stdout
