"""Launch-shape knobs (vx_tuning_*): names, allowed values, defaults,
rejection of unknown knobs and disallowed values.  Host-only calls, no GPU."""
import voxel_b200 as vx

EXPECTED = {"sort.items_u32": 16, "sort.items_u64": 10, "sort.early_counts": 0, "sort.rank_ballots": 0,
            "edit.big_item": 32, "edit.blocks_per_sm": 32,
            "edit.leafparent_blocks": 5, "serve.blocks_per_sm": 4,
            "edit.leafparent_lanes": 4, "edit.small_max_prims": 256,
            "edit.small_blocks_per_sm": 1, "edit.small_max_voxels": 16384,
            "sort.radix_bits": 8, "scan.tile_kb": 32,
            "edit.leafparent_prefetch": 1}


def test_knobs_and_defaults():
    vx.reset_tuning()
    assert vx.tuning() == EXPECTED
    for name, default in EXPECTED.items():
        opts = vx.tuning_options(name)
        assert default in opts and len(opts) >= 2


def test_set_reject_reset():
    try:
        vx.set_tuning("sort.items_u32", 12)
        vx.set_tuning("edit.big_item", 256)
        assert vx.tuning()["sort.items_u32"] == 12
        assert vx.tuning()["edit.big_item"] == 256
        assert vx.lib().vx_tuning_set(b"sort.items_u32", 13) == vx.VX_ERR_INVALID_VALUE
        assert vx.lib().vx_tuning_set(b"no.such.knob", 1) == vx.VX_ERR_INVALID_VALUE
        assert vx.lib().vx_tuning_name(vx.lib().vx_tuning_count()) is None
        assert vx.tuning()["sort.items_u32"] == 12  # a rejected set changes nothing
    finally:
        vx.reset_tuning()
    assert vx.tuning() == EXPECTED


def test_tuning_file_name():
    p = vx.tuning_file("NVIDIA B200")
    assert p.name == "NVIDIA_B200.json" and p.parent.name == "tuning"


def test_committed_b200_settings_are_the_defaults():
    """The autotuner's B200 file holds a valid value for every knob, and the
    library's compiled defaults are that file's choices (a caller that never
    loads the file gets the tuned shapes on B200)."""
    import json
    saved = json.loads(vx.tuning_file("NVIDIA B200").read_text())["knobs"]
    assert set(saved) == set(EXPECTED)
    for name, value in saved.items():
        assert value in vx.tuning_options(name), name
    assert saved == EXPECTED
