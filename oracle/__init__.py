"""CPU oracle of the LATfield2 particle-mesh path -- test infrastructure only."""
