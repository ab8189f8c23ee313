/*
 * TravelDirections (reference: TravelDirections.hpp:46-403), host side.
 * Same enumerator names and values; the 26 neighbour directions are axis-sign
 * triples, so the tables are derived instead of spelled out case by case.
 */
#ifndef CMACIONIZE_TRAVELDIRECTIONS_HPP
#define CMACIONIZE_TRAVELDIRECTIONS_HPP

enum TravelDirection {
  TRAVELDIRECTION_INSIDE = 0,
  TRAVELDIRECTION_CORNER_PPP, TRAVELDIRECTION_CORNER_PPN, TRAVELDIRECTION_CORNER_PNP,
  TRAVELDIRECTION_CORNER_PNN, TRAVELDIRECTION_CORNER_NPP, TRAVELDIRECTION_CORNER_NPN,
  TRAVELDIRECTION_CORNER_NNP, TRAVELDIRECTION_CORNER_NNN,
  TRAVELDIRECTION_EDGE_X_PP, TRAVELDIRECTION_EDGE_X_PN, TRAVELDIRECTION_EDGE_X_NP,
  TRAVELDIRECTION_EDGE_X_NN,
  TRAVELDIRECTION_EDGE_Y_PP, TRAVELDIRECTION_EDGE_Y_PN, TRAVELDIRECTION_EDGE_Y_NP,
  TRAVELDIRECTION_EDGE_Y_NN,
  TRAVELDIRECTION_EDGE_Z_PP, TRAVELDIRECTION_EDGE_Z_PN, TRAVELDIRECTION_EDGE_Z_NP,
  TRAVELDIRECTION_EDGE_Z_NN,
  TRAVELDIRECTION_FACE_X_P, TRAVELDIRECTION_FACE_X_N, TRAVELDIRECTION_FACE_Y_P,
  TRAVELDIRECTION_FACE_Y_N, TRAVELDIRECTION_FACE_Z_P, TRAVELDIRECTION_FACE_Z_N,
  TRAVELDIRECTION_NUMBER
};

namespace TravelDirections {

/* axis signs of a direction: +1 upper face, -1 lower face, 0 not involved */
inline void signs(int direction, int s[3]) {
  static const signed char table[TRAVELDIRECTION_NUMBER][3] = {
      {0, 0, 0},   {1, 1, 1},   {1, 1, -1}, {1, -1, 1}, {1, -1, -1}, {-1, 1, 1},
      {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1},
      {0, -1, -1}, {1, 0, 1},   {1, 0, -1}, {-1, 0, 1}, {-1, 0, -1}, {1, 1, 0},
      {1, -1, 0},  {-1, 1, 0},  {-1, -1, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0},
      {0, -1, 0},  {0, 0, 1},   {0, 0, -1}};
  for (int a = 0; a < 3; ++a) s[a] = table[direction][a];
}

inline int from_signs(int sx, int sy, int sz) {
  for (int d = 0; d < TRAVELDIRECTION_NUMBER; ++d) {
    int s[3];
    signs(d, s);
    if (s[0] == sx && s[1] == sy && s[2] == sz) return d;
  }
  return -1;
}

/* TravelDirections.hpp:89-152 */
inline int output_to_input_direction(int output_direction) {
  if (output_direction < 0 || output_direction >= TRAVELDIRECTION_NUMBER) return -1;
  int s[3];
  signs(output_direction, s);
  return from_signs(-s[0], -s[1], -s[2]);
}

/* TravelDirections.hpp:163-224 */
inline bool is_compatible_output_direction(const double *direction, int output_direction) {
  if (output_direction < 0 || output_direction >= TRAVELDIRECTION_NUMBER) return false;
  int s[3];
  signs(output_direction, s);
  for (int a = 0; a < 3; ++a)
    if ((s[a] > 0 && !(direction[a] > 0.)) || (s[a] < 0 && !(direction[a] < 0.))) return false;
  return true;
}

/* TravelDirections.hpp:235-298 */
inline bool is_compatible_input_direction(const double *direction, int input_direction) {
  if (input_direction < 0 || input_direction >= TRAVELDIRECTION_NUMBER) return false;
  int s[3];
  signs(input_direction, s);
  for (int a = 0; a < 3; ++a)
    if ((s[a] > 0 && !(direction[a] < 0.)) || (s[a] < 0 && !(direction[a] > 0.))) return false;
  return true;
}

/* TravelDirections.hpp:315-403: bits (x_high, x_low, y_high, y_low, z_high, z_low) */
inline int get_output_direction(int mask) {
  if (mask < 0 || mask > 63) return -1;
  int s[3];
  for (int a = 0; a < 3; ++a) {
    const int hi = (mask >> (5 - 2 * a)) & 1, lo = (mask >> (4 - 2 * a)) & 1;
    if (hi && lo) return -1;
    s[a] = hi ? 1 : (lo ? -1 : 0);
  }
  return from_signs(s[0], s[1], s[2]);
}

}  // namespace TravelDirections

#endif
