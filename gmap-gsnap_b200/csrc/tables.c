/*
 * tables.c -- host construction of the substitution and consistency
 * tables, with the values Dynprog_init gives them (src/dynprog.c:1007-1196):
 *
 *   - every letter pair in 'A'..'z' x 'A'..'y' starts as the mismatch
 *     score of its mismatch type (HIGHQ -3, MEDQ -2, LOWQ -1, ENDQ -5;
 *     src/dynprog.h:48-50, src/dynprog.c:103), the second bound being
 *     exclusive as in the reference loop (:1069-1076);
 *   - identical letters 'A'..'Y' (either case) score FULLMATCH 3; U/T 3;
 *     IUPAC two-base codes score HALFMATCH 1 against their bases; three-base
 *     codes, N and X score AMBIGUOUS 3 against their bases; N-N and X-X
 *     score 3 (:1088-1140);
 *   - the cmet / atoi / ttoc modes add one-way entries (:1143-1172);
 *   - consistent_array marks the same pairs per gene strand (:894-970).
 * Scores of a pair are the same for both argument orders except for the
 * one-way entries.  The table contents have to equal the reference's for
 * the scores to be bit-exact; the code that builds them is this library's.
 */
#include <ctype.h>
#include <string.h>
#include "gdp_internal.h"

static void
mark (gdp_tables_t *t, int A, int B, int score, int mode, int oneway, int genestrand) {
  const int a = tolower(A), b = tolower(B);
  const int xs[4] = {a, a, A, A}, ys[4] = {b, B, b, B};
  int k, i;
  for (k = 0; k < 4; k++) {
    int x = xs[k], y = ys[k];
    if (oneway) {
      t->cons[genestrand][x][y] = 1;
    } else if (mode == 0 || mode == 1 || mode == 3 || mode == 5) {   /* *_STRANDED, STANDARD */
      t->cons[0][x][y] = t->cons[0][y][x] = 1;
    } else {
      t->cons[1][x][y] = t->cons[1][y][x] = 1;
      t->cons[2][x][y] = t->cons[2][y][x] = 1;
    }
    for (i = 0; i < 4; i++) {
      t->pd[i][x][y] = (int16_t) score;
      if (!oneway) t->pd[i][y][x] = (int16_t) score;
    }
  }
}

static uint32_t
pack4 (int a, int b, int c, int d) {
  return (uint32_t) (uint8_t) a | ((uint32_t) (uint8_t) b << 8) |
         ((uint32_t) (uint8_t) c << 16) | ((uint32_t) (uint8_t) d << 24);
}

/* The packed class profiles the fill kernels read, from pd. */
void
gdp_tables_derive (gdp_tables_t *t) {
  static const char ACGTN[5] = {'A', 'C', 'G', 'T', 'N'};
  int c1, mt;
  for (mt = 0; mt < 4; mt++) {
    for (c1 = 0; c1 < 128; c1++) {
      int k, q[5], g[5];
      for (k = 0; k < 5; k++) {
        q[k] = t->pd[mt][c1][(int) ACGTN[k]];
        g[k] = t->pd[mt][(int) ACGTN[k]][c1];
      }
      t->profq_lo[mt][c1] = pack4(q[0], q[1], q[2], q[3]);
      t->profq_hi[mt][c1] = pack4(q[4], 0, 0, 0);
      t->profg_lo[mt][c1] = pack4(g[0], g[1], g[2], g[3]);
      t->profg_hi[mt][c1] = pack4(g[4], 0, 0, 0);
    }
  }
}

void
gdp_build_tables (gdp_tables_t *t, int mode) {
  static const int mismatch[4] = {-3, -2, -1, -5};
  static const char two[][2] = {{'R','A'},{'R','G'},{'Y','T'},{'Y','C'},{'W','A'},{'W','T'},
                                {'S','G'},{'S','C'},{'M','A'},{'M','C'},{'K','G'},{'K','T'}};
  static const char three[][2] = {{'H','A'},{'H','T'},{'H','C'},{'B','G'},{'B','C'},{'B','T'},
                                  {'V','G'},{'V','A'},{'V','C'},{'D','G'},{'D','A'},{'D','T'},
                                  {'N','T'},{'N','C'},{'N','A'},{'N','G'},
                                  {'X','T'},{'X','C'},{'X','A'},{'X','G'},{'N','N'},{'X','X'}};
  int c1, c2, i;
  memset(t, 0, sizeof(*t));
  for (i = 0; i < 128; i++) t->nt2int[i] = 4;
  t->nt2int['A'] = t->nt2int['a'] = 0;
  t->nt2int['C'] = t->nt2int['c'] = 1;
  t->nt2int['G'] = t->nt2int['g'] = 2;
  t->nt2int['T'] = t->nt2int['t'] = 3;
  for (c1 = 'A'; c1 <= 'z'; c1++)
    for (c2 = 'A'; c2 < 'z'; c2++)
      for (i = 0; i < 4; i++) t->pd[i][c1][c2] = (int16_t) mismatch[i];
  for (c1 = 'A'; c1 < 'Z'; c1++) mark(t, c1, c1, 3, mode, 0, 0);
  mark(t, 'U', 'T', 3, mode, 0, 0);
  for (i = 0; i < (int) (sizeof(two) / sizeof(two[0])); i++) mark(t, two[i][0], two[i][1], 1, mode, 0, 0);
  for (i = 0; i < (int) (sizeof(three) / sizeof(three[0])); i++) mark(t, three[i][0], three[i][1], 3, mode, 0, 0);
  switch (mode) {
  case 1: mark(t, 'T', 'C', 3, mode, 1, 0); break;                              /* CMET_STRANDED */
  case 2: mark(t, 'T', 'C', 3, mode, 1, 1); mark(t, 'A', 'G', 3, mode, 1, 2); break;  /* CMET_NONSTRANDED */
  case 3: mark(t, 'G', 'A', 3, mode, 1, 0); break;                              /* ATOI_STRANDED */
  case 4: mark(t, 'G', 'A', 3, mode, 1, 1); mark(t, 'C', 'T', 3, mode, 1, 2); break;  /* ATOI_NONSTRANDED */
  case 5: mark(t, 'C', 'T', 3, mode, 1, 0); break;                              /* TTOC_STRANDED */
  case 6: mark(t, 'C', 'T', 3, mode, 1, 1); mark(t, 'G', 'A', 3, mode, 1, 2); break;  /* TTOC_NONSTRANDED */
  default: break;
  }
  gdp_tables_derive(t);
}
