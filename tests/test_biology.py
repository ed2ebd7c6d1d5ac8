"""Biology overrides (astrosim_create_with_biology and friends) on the host side:
the parameter table, the JSON reader's errors, the CLI's --biology flag, and the
oracle's by-name overrides.  Nothing here needs a GPU.
"""
import json
import subprocess

import pytest

import astrosimgpu_cuda_b200 as asg
from oracle import oracle


def test_every_reference_constant_is_named():
    names = asg.biology_names()
    assert len(names) == len(set(names)) == 82
    for n in ("Ca_tot", "SIC_th", "e_Delta_T", "i_tau_syn_in", "stp_U", "sic_interval", "noise_dt",
              "independent_noise", "exc_poiss_rate"):
        assert n in names


def test_defaults_and_overrides():
    assert asg.biology_value("exc_poiss_rate") == 2700.0  # src/astrosim_fused.cu:742-781
    assert asg.biology_value("stp_U") == 0.5
    over = {"exc_poiss_rate": 3000, "stp_enabled": False, "sic_interval": 3}
    assert asg.biology_value("exc_poiss_rate", over) == 3000.0
    assert asg.biology_value("stp_enabled", over) == 0.0
    assert asg.biology_value("sic_interval", json.dumps(over)) == 3.0
    assert asg.biology_value("w_e", "") == 5.0
    assert asg.biology_value("w_e", "  {  } ") == 5.0


@pytest.mark.parametrize("text,needle", [
    ('{"bogus": 1}', "unknown biology parameter 'bogus'"),
    ('{"w_e": true}', "takes a number"),
    ('{"stp_enabled": 2}', "true or false"),
    ('{"sic_interval": 2.5}', "integer"),
    ('{"sic_interval": 0}', "sic_interval"),
    ('{"e_C_m": 0}', "'e_C_m' must be > 0"),
    ('{"d_e": -1}', "'d_e' must be > 0"),
    ('{"exc_noise_std": -1}', ">= 0"),
    ('{"stp_U": 1.5}', "stp_U"),
    ('{"ra_lower": 2.0}', "ra_lower < ra_upper"),
    ('{"w_e": 1, "w_e": 2}', "given twice"),
    ('{"w_e" 1}', "expected ':'"),
    ('{"w_e": 1,}', "quoted name"),
    ('[1]', "expected '{'"),
    ('{"w_e": 1} trailing', "after the closing"),
    ('{"w_e": nan}', "needs a number"),
])
def test_bad_overrides_are_rejected(text, needle):
    with pytest.raises(asg.AstrosimError) as e:
        asg.biology_value("w_e", text)
    assert needle in str(e.value)


def test_cli_rejects_bad_biology_file_before_the_gpu(tmp_path):
    f = tmp_path / "bio.json"
    f.write_text('{"w_e": 4.0, "typo_rate": 1}')
    r = subprocess.run([asg.CLI_PATH, "--n", "100", "--biology", str(f)], capture_output=True, text=True)
    assert r.returncode == 1
    assert "typo_rate" in r.stderr
    r = subprocess.run([asg.CLI_PATH, "--n", "100", "--biology", str(tmp_path / "missing.json")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "cannot read" in r.stderr


def test_oracle_takes_the_same_overrides():
    base = oracle.OracleSim(n_total=500, seed=1, pre_ms=0, sim_ms=5)
    over = oracle.OracleSim(n_total=500, seed=1, pre_ms=0, sim_ms=5, biology={"exc_poiss_rate": 27000.0})
    base.step(50)
    over.step(50)
    assert over.summary()["spikes_total"] > base.summary()["spikes_total"]
    with pytest.raises(ValueError):
        oracle.OracleSim(n_total=500, seed=1, biology={"no_such_constant": 1.0})
