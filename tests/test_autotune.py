"""The autotuner's selection rule (hmat-omp_b200/autotune.py): host logic only."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
spec = importlib.util.spec_from_file_location("autotune", os.path.join(ROOT, "hmat-omp_b200", "autotune.py"))
autotune = importlib.util.module_from_spec(spec)
spec.loader.exec_module(autotune)


def test_select_keeps_only_clear_wins_and_drops_stale_entries():
    base = {"a|f64": ["96,0,0", 10.0], "b|f32": ["64,1,1", 5.0], "c|f64": ["0,0,0", 2.0]}
    runs = [
        {"a|f64": ["32,1,0", 8.0], "b|f32": ["64,1,1", 4.9], "c|f64": ["0,0,0", 1.5]},
        {"a|f64": ["32,1,0", 7.5], "b|f32": ["32,0,1", 4.95]},   # min over repeated choices
        {"z|f64": ["32,0,0", 0.1]},                                # unknown signature: ignored
    ]
    table = {"b|f32": [128, 0, 0], "old|f32": [64, 0, 0]}
    rep = autotune.select(base, runs, 0.03, table)
    assert table["a|f64"] == [32, 1, 0]          # 25% faster: kept
    assert "b|f32" not in table                  # best is within the margin: stale entry dropped
    assert "c|f64" not in table                  # same effective choice as the heuristic
    assert table["old|f32"] == [64, 0, 0]        # signatures not swept stay
    assert "z|f64" not in table
    assert rep["a|f64"] == {"heuristic": ["96,0,0", 10.0], "best": ["32,1,0", 7.5]}


def test_choices_cover_every_tile_width_and_flag():
    assert len(autotune.CHOICES) == 32
    assert {c[0] for c in autotune.CHOICES} == {32, 64, 96, 128}
