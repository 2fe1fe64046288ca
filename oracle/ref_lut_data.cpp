// ref_lut_data.cpp -- TEST INFRASTRUCTURE ONLY (linked into
// oracle/_ref/librise_ref.so by oracle/rise_ref.mk).
//
// The reference library reads its RGB -> spectrum table from three symbols
// that its build generates from the table file (the generated source is not
// part of the reference tree; declarations in
// src/Library/Utilities/Color/RGBToSpectrumTable_LUTData.h):
//   kSpectrumLUTResolution  cells per axis (64),
//   kSpectrumLUTNumFloats   3 * res^3 * 3,
//   kSpectrumLUTFloats      the table body.
// This file defines them from the table the reference's own generator
// (tools/JakobHanikaLUTGen.cpp, run by oracle/Makefile) writes: the body is
// the file after its 20-byte header ('RJHL', version, resolution, channels,
// coefficients), embedded as is with the assembler's .incbin.

#ifndef RISE_LUT_COEFF
#error "RISE_LUT_COEFF must name the generated .coeff file"
#endif

namespace RISE
{
    extern const unsigned int kSpectrumLUTResolution;
    extern const unsigned int kSpectrumLUTNumFloats;
    const unsigned int kSpectrumLUTResolution = 64;
    const unsigned int kSpectrumLUTNumFloats = 3u * 64u * 64u * 64u * 3u;
}

// RISE::kSpectrumLUTFloats (extern const float[] in namespace RISE).
__asm__(
    "  .section .rodata\n"
    "  .balign 16\n"
    "  .globl _ZN4RISE18kSpectrumLUTFloatsE\n"
    "  .type _ZN4RISE18kSpectrumLUTFloatsE, @object\n"
    "_ZN4RISE18kSpectrumLUTFloatsE:\n"
    "  .incbin \"" RISE_LUT_COEFF "\", 20, 9437184\n"
    "  .size _ZN4RISE18kSpectrumLUTFloatsE, 9437184\n"
    "  .previous\n");
