/* The C ABI used from plain C99 (the header must compile as C, not only as C++): CPU-side entry
 * points only, so it runs without a GPU.  Prints "c api ok <sizeof(tc_decode_options)>" on
 * success, exits non-zero with a message on the first mismatch. */
#include <stdio.h>
#include <string.h>

#include "turbo_b200.h"

static int fail(const char* what) {
  fprintf(stderr, "c api check failed: %s (%s)\n", what, tc_last_error());
  return 1;
}

int main(void) {
  const char* msg = "123456789";
  uint8_t bits[72], out[96];
  size_t i;
  int ok = 0;
  uint32_t crc = 0;
  tc_decode_options o;
  tc_segmentation seg;
  uint8_t cb[40], d012[3 * 44];
  int32_t perm[40];
  static uint8_t big[12000];

  if (tc_version() <= 0) return fail("version");
  for (i = 0; i < 72; ++i) bits[i] = (uint8_t)((msg[i / 8] >> (7 - i % 8)) & 1);
  /* TS 36.212 CRC24A of ASCII "123456789": the published check value 0xCDE703 */
  if (tc_crc_append_conv(TC_CONVENTION_3GPP, TC_CRC24A, bits, 72, out) != TC_OK) return fail("crc append");
  for (i = 72; i < 96; ++i) crc = (crc << 1) | out[i];
  if (crc != 0xCDE703u) return fail("crc24a check value");
  if (tc_crc_check_conv(TC_CONVENTION_3GPP, TC_CRC24A, out, 96, &ok) != TC_OK || !ok)
    return fail("crc check");
  /* options: documented defaults */
  if (tc_decode_options_init(&o) != TC_OK) return fail("options init");
  if (o.max_iterations != 8 || o.guard != -1 || o.window != 0 || o.memory != TC_MEM_HOST ||
      o.schedule != TC_SCHEDULE_PLAIN || o.convention != TC_CONVENTION_REFERENCE || o.stream)
    return fail("option defaults");
  /* segmentation sizes of B = 12000 bits: C = 2, K+ = 6080, K- = 6016, 48 filler bits */
  if (tc_segment_transport_block(big, 12000, &seg, NULL, 0) != TC_OK) return fail("segmentation");
  if (seg.c != 2 || seg.c_plus != 1 || seg.c_minus != 1 || seg.k_plus != 6080 ||
      seg.k_minus != 6016 || seg.filler_bits != 48 || seg.l != 24)
    return fail("segmentation sizes");
  /* QPP and encoder on K = 40 */
  if (tc_qpp_permutation(40, perm) != TC_OK || perm[0] != 0) return fail("qpp");
  memset(cb, 0, sizeof cb);
  cb[3] = 1;
  if (tc_turbo_encode_conv(TC_CONVENTION_3GPP, 40, 0, cb, d012) != TC_OK) return fail("encode");
  if (d012[3] != 1) return fail("systematic bit");
  /* errors come back as status codes with a message */
  if (tc_qpp_permutation(44, perm) != TC_ERR_OUT_OF_RANGE) return fail("K=44 not refused");
  if (strlen(tc_last_error()) == 0) return fail("no error message");
  printf("c api ok %u\n", (unsigned)sizeof(tc_decode_options));
  return 0;
}
