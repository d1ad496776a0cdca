"""The render command's argument handling (src/app/render_cli.cpp:46-121): option errors are
reported before any scene is loaded, so they run without a GPU."""

import pytest

from minirender_b200 import render_cli


@pytest.mark.parametrize("argv, message", [
    ([], "Usage: --render"),
    (["scene.json"], "Usage: --render"),
    (["scene.json", "out", "--spp"], "missing its value: --spp"),
    (["scene.json", "out", "--width", "abc"], "Invalid number: abc"),
    (["scene.json", "out", "--height", "-4"], "Invalid number: -4"),
    (["scene.json", "out", "--mode", "path"], "Sampling mode must be bsdf, light or mis"),
    (["scene.json", "out", "--integrator", "sppm"], "SPPM is not supported"),
    (["scene.json", "out", "--photons", "1000"], "SPPM is not supported"),
    (["scene.json", "out", "--exposure", "65"], "Exposure must be finite"),
    (["scene.json", "out", "--exposure", "nan"], "Exposure must be finite"),
    (["scene.json", "out", "--frobnicate", "1"], "Unknown render option: --frobnicate"),
])
def test_option_errors(argv, message):
    with pytest.raises(ValueError, match=message.replace("(", r"\(")):
        render_cli.run(argv)


def test_main_prints_the_error_and_returns_one(capsys, monkeypatch):
    monkeypatch.setattr("sys.argv", ["render_cli", "--render", "scene.json", "out", "--mode", "x"])
    assert render_cli.main() == 1
    assert "error: Sampling mode must be bsdf, light or mis" in capsys.readouterr().err


def test_trace_normals_needs_two_paths(capsys, monkeypatch):
    monkeypatch.setattr("sys.argv", ["render_cli", "--trace-normals", "scene.json"])
    assert render_cli.main() == 1
    assert "Usage: --trace-normals" in capsys.readouterr().err


def test_path_integrator_is_accepted_before_the_scene_is_read(tmp_path):
    # `--integrator path` is the default integrator: parsing goes on to the scene file, whose
    # absence is the first error.
    with pytest.raises((OSError, ValueError)) as error:
        render_cli.run([str(tmp_path / "missing.json"), "out", "--integrator", "path",
                        "--no-rr", "--rr-depth", "2", "--seed", "5", "--threads", "2",
                        "--tile", "16", "--batch", "4", "--exposure", "-1.5"])
    assert "SPPM" not in str(error.value)
