"""The generate command (ssms/cli/generate.py): YAML -> configs and the
output folder layout on CPU; files written through the GPU pipeline."""

import io
import logging
import pickle

import numpy as np
import pytest

from ssms_b200 import cli

YAML = """
MODEL: 'angle'
GENERATOR_APPROACH: 'lan'
PIPELINE:
  N_PARAMETER_SETS: 6
  N_SUBRUNS: 2
  N_CPUS: 3
SIMULATOR:
  N_SAMPLES: 2000
  DELTA_T: 0.002
TRAINING:
  N_SAMPLES_PER_PARAM: 40
ESTIMATOR:
  TYPE: 'KDE'
"""


def test_yaml_config_is_merged_into_the_generator_defaults(tmp_path):
    cfg = cli.collect_data_generator_config(io.StringIO(YAML), base_path=tmp_path)
    dc, mc = cfg["data_config"], cfg["model_config"]
    assert dc["model"] == "angle" and mc["name"] == "angle"
    assert dc["generator_approach"] == "lan" and dc["cpn_only"] is False
    assert dc["output"]["folder"] == str(tmp_path / "data/training_data/lan/training_data_n_samples_2000_dt_0.002/angle")
    assert dc["output"]["pickle_protocol"] == 4  # untouched defaults survive the merge
    assert dc["pipeline"]["n_parameter_sets"] == 6 and dc["pipeline"]["n_subruns"] == 2
    assert dc["pipeline"]["n_cpus"] == 3
    assert "simulation_filters" in dc["pipeline"]
    assert dc["simulator"]["n_samples"] == 2000 and dc["simulator"]["delta_t"] == 0.002
    assert dc["simulator"]["max_t"] == 20.0
    assert dc["training"]["n_samples_per_param"] == 40
    assert dc["estimator"]["type"] == "kde"


def test_default_yaml_and_cli_overrides(tmp_path):
    logger = logging.getLogger("test")
    cfg, sha = cli.load_config(None, tmp_path, "KDE", logger, n_cpus=2)
    assert sha is not None and len(sha) == 64
    assert cfg["data_config"]["model"] == "ddm"
    assert cfg["data_config"]["estimator_type"] == "kde"
    assert cfg["data_config"]["pipeline"]["n_cpus"] == 2
    assert cfg["data_config"]["pipeline"]["n_parameter_sets"] == 100


@pytest.mark.parametrize("value,expected", [(None, None), ("all", "all"), ("4", 4), (2, 2), (3.0, 3)])
def test_n_cpus_accepts_positive_integers_and_all(value, expected):
    assert cli.parse_n_cpus(value) == expected


@pytest.mark.parametrize("value", [0, "0", -1, True, 2.5, "many"])
def test_n_cpus_rejects_everything_else(value):
    with pytest.raises(cli.ConfigError):
        cli.parse_n_cpus(value)


def test_bad_pipeline_n_cpus_in_yaml_is_rejected(tmp_path):
    with pytest.raises(cli.ConfigError, match="PIPELINE.N_CPUS"):
        cli.collect_data_generator_config(io.StringIO(YAML.replace("N_CPUS: 3", "N_CPUS: 0")), base_path=tmp_path)


def test_config_can_be_saved(tmp_path):
    cfg = cli.make_data_generator_configs(model="ddm", data_generator_nested_dict={"training": {"n_samples_per_param": 7}},
                                          save_name="cfg.pickle", save_folder=tmp_path)
    with open(tmp_path / "cfg.pickle", "rb") as f:
        back = pickle.load(f)
    assert back["data_config"]["training"]["n_samples_per_param"] == 7
    assert back["data_config"] == cfg["data_config"]


def test_unknown_estimator_exits_with_error(tmp_path):
    y = tmp_path / "c.yaml"
    y.write_text(YAML)
    assert cli.main(["--config-path", str(y), "--output", str(tmp_path), "-e", "pyddm"]) == 1


@pytest.mark.gpu
def test_generate_writes_training_files(cuda, tmp_path):
    y = tmp_path / "c.yaml"
    y.write_text(YAML)
    assert cli.main(["--config-path", str(y), "--output", str(tmp_path), "-n", "2", "--seed", "5"]) == 0
    folder = tmp_path / "data/training_data/lan/training_data_n_samples_2000_dt_0.002/angle"
    files = sorted(folder.glob("*.pickle"))
    assert len(files) == 2
    with open(files[0], "rb") as f:
        data = pickle.load(f)
    P = 5  # angle: v, a, z, t, theta
    assert data["lan_data"].shape == (6 * 40, P + 2) and data["lan_labels"].shape == (6 * 40,)
    assert data["lan_data"].dtype == np.float32
    assert data["cpn_labels"].shape == (6, 1) and data["binned_128"].shape == (6, 128, 2)
    assert np.all(np.isfinite(data["lan_labels"]))
    assert data["generator_config"]["simulator"]["delta_t"] == 0.002
    assert data["model_config"]["name"] == "angle"
    # a dry run writes nothing
    assert cli.main(["--config-path", str(y), "--output", str(tmp_path), "--dry-run", "--backend", "per_set"]) == 0
    assert len(sorted(folder.glob("*.pickle"))) == 2
