/*
 * The reference's own main() (sp_3d_ns.cxx:442-657, compiled as
 * kapsel_reference_main by oracle/Makefile) as a program.  TEST
 * INFRASTRUCTURE ONLY: linked once with the reference objects alone and once
 * with the GPU shims (kapsel_old_b200/shim) in place of the functions they
 * replace, so that the two runs of the same input can be compared.
 */
int kapsel_reference_main(int argc, char *argv[]);

int main(int argc, char *argv[]) { return kapsel_reference_main(argc, argv); }
