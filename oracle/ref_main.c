/* main of the reference's program built from its own objects (its Main.c is
 * compiled with main renamed to sfr3d_ref_main): oracle/Makefile `dropin`. */
int sfr3d_ref_main(int argc, char **argv);

int main(int argc, char **argv) { return sfr3d_ref_main(argc, argv); }
