/* palette_dump.c -- TEST INFRASTRUCTURE: writes the colour tables of the
 * reference's ppm output (src/palette.h, included from the reference tree at
 * build time) as text lines "<name> v0 .. v767", each value printed with
 * enough digits to read back as the same float.  oracle/build_ref.py runs it
 * into oracle/_ref/palettes.txt, the palette file the ppm parity tests hand
 * to the command-line driver on machines without the reference tree. */
#include <stdio.h>

#include "palette.h"

int main(void) {
  int i, k;
  for (i = 0; rgb[i].name && rgb[i].rgb; i++) {
    printf("%s", rgb[i].name);
    for (k = 0; k < 256 * 3; k++) printf(" %.9g", (double)rgb[i].rgb[k]);
    printf("\n");
  }
  return 0;
}
