"""Environments by name (src/microcosmos/gym/registry.py:10-34)."""
from __future__ import annotations

from .base import Environment
from .envs import LineEnv, LineRingEnv, MultiAgentEnv, RandomFoodLineEnv, RingEnv, TadpoleEnv

_REGISTRY: dict[str, type[Environment]] = {
    "line": LineEnv,
    "line-random-food": RandomFoodLineEnv,
    "line-ring": LineRingEnv,
    "multi-agent": MultiAgentEnv,
    "ring": RingEnv,
    "tadpole": TadpoleEnv,
}


def make(name: str, **kwargs) -> Environment:
    """Build a predefined environment by name; extra kwargs go to its constructor."""
    if name not in _REGISTRY:
        raise ValueError(f"unknown env {name!r}; choices: {sorted(_REGISTRY)}")
    return _REGISTRY[name](**kwargs)


def registered_envs() -> list[str]:
    return sorted(_REGISTRY)
