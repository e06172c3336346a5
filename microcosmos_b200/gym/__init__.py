"""Gym environments around the device rollout (src/microcosmos/gym/): the reference's
pure-functional ``reset``/``step`` interface, its predefined environments and registry,
and ``BatchedEnv`` -- many environments stepped together in one launch sequence (the
reference's ``jax.vmap`` over ``step``)."""
from . import topology
from .base import Environment, EnvState
from .batched import BatchedEnv
from .envs import (CreatureTopology, LineEnv, LineRingEnv, LineTopology, MultiAgentEnv, RandomFoodLineEnv, RingEnv,
                   RingTopology, TadpoleEnv)
from .registry import make, registered_envs

__all__ = ["Environment", "EnvState", "BatchedEnv", "CreatureTopology", "LineEnv", "LineRingEnv", "LineTopology",
           "MultiAgentEnv", "RandomFoodLineEnv", "RingEnv", "RingTopology", "TadpoleEnv", "make", "registered_envs", "topology"]
