"""CPU oracle for the GFDL microphysics path. Test infrastructure only: the
product package never imports it."""
