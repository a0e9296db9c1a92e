"""``generate``: training-data files from a YAML configuration, on the GPU.

The reference's data-generation command (ssms/cli/generate.py): the same YAML
keys (MODEL, GENERATOR_APPROACH, PIPELINE, SIMULATOR, TRAINING, ESTIMATOR),
the same output folder layout
(``<output>/data/training_data/<approach>/training_data_n_samples_<n>_dt_<dt>/<model>``),
the same config merge and ``--n-cpus`` validation, and one pickle per file
written by ``TrainingDataGenerator``.  ``--backend`` picks the GPU pipeline:
``batched`` (thousands of parameter sets per device step, the default) or
``per_set`` (the reference's one-set-at-a-time pipeline over the GPU simulator
and KDE).  The reference's MLflow logging is not part of this package.

    python -m ssms_b200.cli --config-path cfg.yaml --output out -n 2
"""

from __future__ import annotations

import argparse
import hashlib
import logging
import pickle
from collections import namedtuple
from pathlib import Path
from pprint import pformat
from typing import Any

import yaml

from .config import ModelConfigBuilder
from .dataset_generators import TrainingDataGenerator, get_default_generator_config

DEFAULT_CONFIG = Path(__file__).resolve().parent / "config_data_generation.yaml"


class ConfigError(ValueError):
    """A configuration value the command rejects (the reference raises typer.BadParameter)."""


def make_data_generator_configs(model="ddm", generator_approach="lan", data_generator_nested_dict=None,
                                model_config_arg_dict=None, save_name=None, save_folder="") -> dict[str, Any]:
    """{"model_config", "data_config"}: the model's config and the approach's
    default generator config with the given sections merged in
    (ssms/cli/generate.py:22-62); pickled to save_folder/save_name if asked."""
    model_config = ModelConfigBuilder.from_model(model)
    data_config = get_default_generator_config(generator_approach, model=model)
    for section, values in (data_generator_nested_dict or {}).items():
        if section in data_config and isinstance(values, dict):
            data_config[section].update(values)
        else:
            data_config[section] = values
    model_config.update(model_config_arg_dict or {})
    data_config["generator_approach"] = generator_approach
    config_dict = {"model_config": model_config, "data_config": data_config}
    if save_name:
        Path(save_folder).mkdir(parents=True, exist_ok=True)
        with open(Path(save_folder) / save_name, "wb") as f:
            pickle.dump(config_dict, f)
    return config_dict


def parse_dict_as_namedtuple(d: dict, to_lowercase: bool = True):
    """A YAML mapping as attribute-access records: every mapping (nested ones
    too) becomes a namedtuple with the keys as fields, lower-cased unless
    ``to_lowercase`` is false, so ``cfg.simulator.n_samples`` reads the
    SIMULATOR section's n_samples; other values are kept as they are."""
    if not isinstance(d, dict):
        return d
    fields = {(k.lower() if to_lowercase else k): parse_dict_as_namedtuple(v, to_lowercase) for k, v in d.items()}
    return namedtuple("Config", list(fields))(*fields.values())


def _make_data_folder_path(base_path, basic_config) -> Path:
    return Path(Path(base_path) / "data/training_data" / basic_config.generator_approach
                / f"training_data_n_samples_{basic_config.simulator.n_samples}_dt_{basic_config.simulator.delta_t}"
                / basic_config.model)


def get_basic_config_from_yaml(yaml_config_path, base_path=None):
    """(namedtuple of the YAML, training-data folder under base_path)."""
    if hasattr(yaml_config_path, "read"):
        raw = yaml.safe_load(yaml_config_path)
    else:
        with open(yaml_config_path, "rb") as f:
            raw = yaml.safe_load(f)
    bc = parse_dict_as_namedtuple(raw)
    return bc, _make_data_folder_path(base_path=base_path, basic_config=bc)


def parse_n_cpus(value, source: str = "--n-cpus"):
    """A positive integer or 'all' (None passes through); anything else --
    0, booleans, fractional floats, other strings -- is rejected."""
    if value is None or value == "all":
        return value
    if isinstance(value, bool):
        raise ConfigError(f"{source} must be an integer or 'all', got {value!r}.")
    if isinstance(value, float) and not value.is_integer():
        raise ConfigError(f"{source} must be a whole number or 'all', got {value!r}.")
    try:
        parsed = int(value)
    except (TypeError, ValueError):
        raise ConfigError(f"{source} must be a positive integer or 'all', got {value!r}.") from None
    if parsed < 1:
        raise ConfigError(f"{source} must be >= 1, got {parsed}.")
    return parsed


def collect_data_generator_config(yaml_config_path=None, base_path=None, extra_configs=None) -> dict[str, Any]:
    """The generator and model configs a YAML file describes
    (ssms/cli/generate.py:150-211): every PIPELINE key, SIMULATOR n_samples
    and delta_t, TRAINING n_samples_per_param, ESTIMATOR type, and the output
    folder under base_path."""
    bc, folder = get_basic_config_from_yaml(yaml_config_path, base_path=base_path)
    nested = {"output": {"folder": str(folder)}, "model": bc.model,
              "cpn_only": bc.generator_approach == "cpn"}
    if hasattr(bc, "pipeline"):
        pipeline = bc.pipeline._asdict()
        if "n_cpus" in pipeline:
            pipeline["n_cpus"] = parse_n_cpus(pipeline["n_cpus"], source="PIPELINE.N_CPUS")
        nested["pipeline"] = pipeline
    if hasattr(bc, "simulator"):
        nested["simulator"] = {"n_samples": bc.simulator.n_samples, "delta_t": bc.simulator.delta_t}
    if hasattr(bc, "training"):
        nested["training"] = {"n_samples_per_param": bc.training.n_samples_per_param}
    if hasattr(bc, "estimator"):
        nested["estimator"] = {"type": bc.estimator.type.lower()}
    return make_data_generator_configs(model=bc.model, generator_approach=bc.generator_approach,
                                       data_generator_nested_dict=nested, model_config_arg_dict=extra_configs)


def load_config(config_path, output, estimator_type, logger, n_cpus=None) -> tuple[dict, str | None]:
    """(config dict, sha256 of the YAML that drove it); the packaged default
    YAML when config_path is None; CLI overrides of the estimator type and
    n_cpus applied last."""
    if config_path is None:
        logger.warning("No config path provided, using default configuration.")
        config_path = DEFAULT_CONFIG
    try:
        sha = hashlib.sha256(Path(config_path).read_bytes()).hexdigest()
    except OSError:
        sha = None
    config_dict = collect_data_generator_config(yaml_config_path=config_path, base_path=output)
    if estimator_type is not None:
        logger.info("Overriding estimator_type from CLI: %s", estimator_type)
        config_dict["data_config"]["estimator_type"] = estimator_type.lower()
    if n_cpus is not None:
        config_dict["data_config"].setdefault("pipeline", {})["n_cpus"] = n_cpus
        logger.info("Overriding n_cpus from CLI: %s", n_cpus)
    logger.debug("GENERATOR CONFIG\n%s", pformat(config_dict["data_config"]))
    return config_dict, sha


def _estimator_type(config_dict: dict) -> str:
    dc = config_dict["data_config"]
    return str(dc.get("estimator_type") or dc.get("estimator", {}).get("type", "kde")).lower()


def generate_data(config_dict: dict, n_files: int, dry_run: bool, logger, backend: str = "batched",
                  seed: int | None = None) -> tuple[list[Path], Path]:
    """Write n_files training-data pickles (or, dry run, generate one set of
    records without saving); returns (new files, output folder)."""
    gen = TrainingDataGenerator(config=config_dict["data_config"], model_config=config_dict["model_config"],
                                backend=backend)
    folder = Path(config_dict["data_config"]["output"]["folder"])
    existing = set(folder.rglob("*.pickle")) if folder.exists() else set()
    if dry_run:
        gen.generate_data_training(save=False, seed=seed)
        logger.info("DRY RUN: pipeline ran; would write %d file(s) to %s", n_files, folder)
        return [], folder
    for i in range(n_files):
        gen.generate_data_training(save=True, seed=None if seed is None else seed + i)
    new = sorted(set(folder.rglob("*.pickle")) - existing) if folder.exists() else []
    logger.info("Newly generated files: %d", len(new))
    return new, folder


def build_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="generate", description="Generate LAN training data on the GPU.")
    ap.add_argument("--config-path", type=Path, default=None, help="Path to the YAML configuration file.")
    ap.add_argument("--output", type=Path, required=True, help="Path to the output directory.")
    ap.add_argument("--n-files", "-n", type=int, default=1, help="Number of files to generate.")
    ap.add_argument("--n-cpus", default=None, help="Positive integer or 'all' (overrides PIPELINE.N_CPUS).")
    ap.add_argument("--dry-run", action="store_true", help="Validate the pipeline without saving any data.")
    ap.add_argument("--estimator-type", "-e", default=None, help="Likelihood estimator type ('kde').")
    ap.add_argument("--backend", choices=("batched", "per_set"), default="batched",
                    help="GPU pipeline: batched parameter sets (default) or one set at a time.")
    ap.add_argument("--seed", type=int, default=None, help="Seed of the first file (default: random).")
    ap.add_argument("--log-level", default="WARNING", help="Logging level.")
    return ap


def main(argv=None) -> int:
    ap = build_parser()
    args = ap.parse_args(argv)
    logging.basicConfig(level=args.log_level.upper(), format="%(asctime)s - %(levelname)s - %(message)s")
    logger = logging.getLogger("ssms_b200.generate")
    if args.n_files < 1:
        ap.error("--n-files must be >= 1")
    try:
        n_cpus = parse_n_cpus(args.n_cpus)
        config_dict, _ = load_config(args.config_path, args.output, args.estimator_type, logger, n_cpus=n_cpus)
    except ConfigError as e:
        ap.error(str(e))
    if _estimator_type(config_dict) != "kde":
        logger.error("estimator type %r is not available: this package builds the KDE estimator",
                     _estimator_type(config_dict))
        return 1
    generate_data(config_dict, args.n_files, args.dry_run, logger, backend=args.backend, seed=args.seed)
    logger.info("DRY RUN complete - no data was saved" if args.dry_run else "Data generation finished")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
