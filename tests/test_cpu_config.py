"""The batched path's run-time knobs (anionpy_b200/_config.py): defaults are
off, the environment wins over IONP_CONFIG, malformed values raise."""
import json

import pytest

from anionpy_b200._config import settings


def test_defaults_are_off():
    assert settings({}) == {"batch_schedule": None, "batch_picker": "off"}


def test_environment_and_file(tmp_path):
    p = tmp_path / "ionp.json"
    p.write_text(json.dumps({"batch_schedule": 24, "batch_picker": "stream"}))
    assert settings({"IONP_CONFIG": str(p)}) == {"batch_schedule": 24, "batch_picker": "stream"}
    env = {"IONP_CONFIG": str(p), "IONP_BATCH_SCHEDULE": "3", "IONP_BATCH_PICKER": "AUTOTUNE"}
    assert settings(env) == {"batch_schedule": 3, "batch_picker": "autotune"}


@pytest.mark.parametrize("env", [{"IONP_BATCH_SCHEDULE": "48"}, {"IONP_BATCH_SCHEDULE": "x"},
                                 {"IONP_BATCH_PICKER": "mlp"}, {"IONP_BATCH_SCHEDULE": "-1"}])
def test_malformed_values_raise(env):
    with pytest.raises(ValueError):
        settings(env)


def test_config_must_be_an_object(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text("[1, 2]")
    with pytest.raises(ValueError):
        settings({"IONP_CONFIG": str(p)})
