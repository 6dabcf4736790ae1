"""Test-side access to the package's seeded configurations (femtools.jl_b200/configs.py)."""
from conftest import fem

StokesCase = fem.configs.StokesCase
vep_layers_case = fem.configs.vep_layers_case
inclusion_2d_case = fem.configs.inclusion_2d_case
random_state_case = fem.configs.random_state_case
