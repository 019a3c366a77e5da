/* The C ABI header compiles as strict C99 and links against the library;
 * run without a GPU it reports the version and a device count. */
#include <stdio.h>
#include <string.h>

#include "sparkit_b200.h"

int main(void) {
  int count = -1;
  sk_matrix A = NULL;
  sk_summary s;
  memset(&s, 0, sizeof s);
  if (strstr(sk_version(), "sm_100a") == NULL) return 1;
  if (sk_device_count(&count) != SK_OK || count < 0) return 2;
  if (count == 0) {
    long long rp[2] = {0, 1}, ci[1] = {0};
    double v[1] = {2.0};
    if (sk_csr_create(&A, 1, 1, (const int64_t*)rp, (const int64_t*)ci, v, SK_F64) != SK_NO_DEVICE) return 3;
  }
  printf("c99 header ok: %s, %d device(s), summary %zu bytes\n", sk_version(), count, sizeof s);
  return 0;
}
