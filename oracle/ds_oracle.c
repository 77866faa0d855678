/* TEST INFRASTRUCTURE ONLY. CPU restatement of the sub-media binning of
 * +MCmatlab/src/getDownsampledParamVals.c:54-202 (greedy farthest-point downsampling of
 * (mua, mus, g) triples to nb representatives, each point labelled with its nearest one), written
 * as the plain serial algorithm with its exact arithmetic:
 *   - per row, extremes and the sum in float, in point order; rows that take one value drop out;
 *   - coordinates are the values times the reciprocal of the row's range (float): the reference
 *     divides, but its own build flags (-Ofast, getDownsampledParamVals.c:22-40) turn the
 *     loop-invariant division into a reciprocal and a multiply, and its outputs agree with this
 *     form bit for bit (tests/test_downsample_oracle.py), not with the division;
 *   - a squared distance accumulates in float, each term (a - b)^2 formed and added in double;
 *   - the first representative is the point farthest from the mean (sum / range / n), the second
 *     the point farthest from the first; thereafter every new representative updates the nearest
 *     distances and labels in one scan that also tracks a running farthest index, which starts
 *     from the index the previous scan ended with and compares against the current contents of
 *     the distance array (possibly not yet updated in this scan); the next representative is
 *     that index unless point 0 is at least as far;
 *   - representatives are scaled back by the range; rows that do not vary take the first
 *     point's value.
 * par is [3 x n] (mua, mus, g per point), out [3 x nb], bin [n] 1-based. */
#include <stdint.h>
#include <stdlib.h>

static float add_sq(float acc, float diff) { return (float)((double)acc + (double)diff * (double)diff); }

int orc_downsample(const float *par, long n, int nb, float *out, uint8_t *bin) {
  if (n < 1 || nb < 1 || nb > 255) return 1;
  float mx[3], mn[3], sm[3], range[3], mterm[3];
  int vary[3], rows = 0;
  for (int c = 0; c < 3; c++) mx[c] = mn[c] = sm[c] = par[c];
  for (long i = 1; i < n; i++)
    for (int c = 0; c < 3; c++) {
      float v = par[3 * i + c];
      if (v > mx[c]) mx[c] = v;
      if (v < mn[c]) mn[c] = v;
      sm[c] += v;
    }
  for (int c = 0; c < 3; c++) {
    vary[c] = mx[c] != mn[c];
    range[c] = mx[c] - mn[c];
    volatile float q = sm[c] / range[c];
    mterm[c] = q / (float)n;
    rows += vary[c];
  }
  float *nv = malloc(sizeof(float) * (size_t)(rows ? rows : 1) * (size_t)n);
  float *d = calloc((size_t)n, sizeof(float));
  float *cen = malloc(sizeof(float) * (size_t)(rows ? rows : 1) * (size_t)nb);
  if (!nv || !d || !cen) return 2;
  long far = 0;
  for (long i = 0; i < n; i++) {
    int r = 0;
    for (int c = 0; c < 3; c++)
      if (vary[c]) {
        nv[rows * i + r] = par[3 * i + c] * (1.0f / range[c]);
        d[i] = add_sq(d[i], nv[rows * i + r] - mterm[c]);
        r++;
      }
    if (d[i] > d[far]) far = i;
  }
  for (int r = 0; r < rows; r++) cen[r] = nv[rows * far + r];
  far = 0;
  for (long i = 0; i < n; i++) {
    d[i] = 0.f;
    for (int r = 0; r < rows; r++) d[i] = add_sq(d[i], nv[rows * i + r] - cen[r]);
    bin[i] = 1;
    if (d[i] > d[far]) far = i;
  }
  long carried = 0;
  for (int j = 1; j < nb; j++) {
    for (int r = 0; r < rows; r++) cen[rows * j + r] = nv[rows * far + r];
    for (long k = 0; k < n; k++) {
      float dk = 0.f;
      for (int r = 0; r < rows; r++) dk = add_sq(dk, nv[rows * k + r] - cen[rows * j + r]);
      if (dk < d[k]) {
        d[k] = dk;
        bin[k] = (uint8_t)(j + 1);
      }
      if (d[k] > d[carried]) carried = k;
    }
    far = d[carried] > d[0] ? carried : 0;
  }
  for (int i = 0; i < nb; i++) {
    int r = 0;
    for (int c = 0; c < 3; c++) {
      out[3 * i + c] = vary[c] ? cen[rows * i + r] * range[c] : par[c];
      r += vary[c];
    }
  }
  free(nv);
  free(d);
  free(cen);
  return 0;
}
