"""CPU oracle of the photon-transport path (test infrastructure only)."""
