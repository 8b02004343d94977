"""The perft_gpu program without a GPU: usage, the UCI handshake and position
handling, and a clean failure (exit 1, a status message) where the engine is
needed.  The counting paths run in the gpu tests."""
import os
import subprocess

import pytest

from tests._oracle import ROOT

CLI = os.path.join(ROOT, "perft_gpu_b200", "perft_gpu")


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        from perft_gpu_b200 import build
        build.build()
    return CLI


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


def test_usage(cli):
    r = subprocess.run([cli, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "Usage perft_gpu <fen> <depth>" in r.stdout


def test_uci_handshake_and_positions(cli):
    script = ("uci\nisready\nposition startpos moves e2e4 e7e5 g1f3\nd\n"
              "position startpos moves e2e5\nposition fen not-a-fen\nbogus\nquit\n")
    r = subprocess.run([cli, "--uci"], input=script, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    out = r.stdout.splitlines()
    assert "uciok" in out and "readyok" in out
    assert "Fen: rnbqkbnr/pppp1ppp/8/4p3/4P3/5N2/PPPP1PPP/RNBQKB1R b KQkq - 0 1" in out
    assert "info string illegal move e2e5" in out
    assert "info string bad fen" in out
    assert "info string unknown command bogus" in out


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present; covered by the gpu tests")
def test_fails_cleanly_without_gpu(cli, tmp_path):
    r = subprocess.run([cli, "startpos", "3"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "perft_init failed" in r.stderr
    r = subprocess.run([cli, "--uci"], input="go perft 2\nquit\n", capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "info string no GPU engine" in r.stdout
    bad = subprocess.run([cli, "nonsense/fen w - -", "3"], capture_output=True, text=True, timeout=60)
    assert bad.returncode == 2 and "bad FEN" in bad.stderr


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present; covered by the gpu tests")
def test_sharded_deep_fails_cleanly_without_gpu(cli):
    """With <gpus> above 1 the deep depths run in shard processes; when they
    cannot start an engine the parent reports the failure instead of a count."""
    env = dict(os.environ, PERFT_DIVIDED_DEPTH="2")
    r = subprocess.run([cli, "startpos", "3", "2"], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 1
    assert "perft(3) failed" in r.stderr and "Perft(03)" not in r.stdout
