/*
 * coulomb_oracle_fp32.c -- FP32 restatement of KTT's known-answer generator.
 *
 * TEST INFRASTRUCTURE ONLY (see coulomb_oracle.c).
 *
 * Restates Examples/JSON/generate-coulomb-output.c:5-38 of KTT 2.1.0: the
 * deterministic 64-atom system of the JSON tuning script
 * (Examples/JSON/CoulombSum3d.json:96-136) and its 256^3 FP32 map written to
 * Coulomb3d.bin.  The arithmetic is kept in the same order, with the same
 * operations (float products, float differences, left-to-right sum of
 * squares, sqrtf, one division, accumulation into the zero-initialised grid),
 * so that, compiled with -ffp-contract=off like the reference recipe in
 * oracle/Makefile, it reproduces the reference's output bit for bit.  That
 * bit-exact match is what pins this restatement; the FP64 oracle is then
 * checked against the same file within KTT's 0.01 tolerance.
 */
#include <math.h>
#include <stdint.h>

#define ORACLE_API __attribute__((visibility("default")))

/* Atom i of the known-answer system: generate-coulomb-output.c:15-20. */
ORACLE_API void oracle_kat_atoms(int n, float* xyzq)
{
    for (int i = 0; i < n; i++) {
        xyzq[i * 4 + 0] = 1.0f + (float)i * 0.1f;
        xyzq[i * 4 + 1] = 1.0f + (float)i * 0.15f;
        xyzq[i * 4 + 2] = 1.0f + (float)i * 0.2f;
        xyzq[i * 4 + 3] = (float)(i % 10) * 0.1f;
    }
}

/*
 * FP32 map, generate-coulomb-output.c:22-31: grid[z][y][x] += q / sqrtf(r^2)
 * over atoms in order.  Only slices [z0, z1) are computed (the full map is
 * z0=0, z1=cells) so a test can check a band of slices quickly.  out holds
 * (z1-z0)*cells*cells floats.
 */
ORACLE_API void oracle_kat_fp32(const float* atoms, int a, float gs, int cells, int z0, int z1, float* out)
{
    for (int z = z0; z < z1; z++)
        for (int y = 0; y < cells; y++)
            for (int x = 0; x < cells; x++) {
                float g = 0.0f;
                for (int at = 0; at < a; at++) {
                    float dx = (float)x * gs - atoms[at * 4 + 0];
                    float dy = (float)y * gs - atoms[at * 4 + 1];
                    float dz = (float)z * gs - atoms[at * 4 + 2];
                    float e = atoms[at * 4 + 3] / sqrtf(dx * dx + dy * dy + dz * dz);
                    g += e;
                }
                out[((int64_t)(z - z0) * cells + y) * cells + x] = g;
            }
}
