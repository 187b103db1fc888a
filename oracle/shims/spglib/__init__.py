"""Oracle shim: the reference imports ``spglib`` unconditionally
(hafnium/symmetry/space_group.py:31) but the molecular DF-RHF path never calls
it. Test infrastructure only."""
