/*
 * Prints, as JSON, the offset of every member of the boundary structs as the
 * REFERENCE's headers lay them out (include/Particles.h, EMfield.h, Grid.h,
 * InterpDensSpecies.h, InterpDensNet.h, Parameters.h). TEST INFRASTRUCTURE ONLY: run by
 * tests/golden/make_golden.py to produce tests/golden/abi_layout.json.
 */
#include <cstddef>
#include <cstdio>
#include <string>

#include "EMfield.h"
#include "Grid.h"
#include "InterpDensNet.h"
#include "InterpDens_aux.h"
#include "InterpDensSpecies.h"
#include "Parameters.h"
#include "Particles.h"
#include "../sputnipic_b200/csrc/abi_layout_fields.h"

int main() {
  std::string out = "{\n";
  SPB_LAYOUT_ALL(SPB_LAYOUT_EMIT_MEMBER)
  SPB_LAYOUT_STRUCTS(SPB_LAYOUT_EMIT_SIZE)
  out += "\"end\": 0\n}\n";
  std::fputs(out.c_str(), stdout);
  return 0;
}
