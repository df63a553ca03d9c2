"""The script-level front-end of the reference (cfms_tomo/shell_test): mesh
loading into the C-ABI arrays and the ``tomoSh_Cpp`` runner used by
TSE_TomoSh1.py."""
