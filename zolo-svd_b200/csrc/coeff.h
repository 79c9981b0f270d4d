// Host scalar routines of the polar iterations (see coeff.cpp).
#pragma once

namespace zolo {

double eps_precision();
void mellipke(double alpha, double tol, double* k, double* e);
void mellipj(double u, double alpha, double tol, double* sn, double* cn, double* dn);
int choosem(double con);
// coeff[0:2rk] = c_i ; coeff[2rk+i] = reference weight (a_i = -coeff[2rk+i])
void compute_coeff(double con, double tol, int rk, double* coeff);
// The same coefficients from the complementary modulus 1/CON used directly (accurate at any
// CON; compute_coeff follows the reference, alpha = acos(1/CON), exact only to ~1e-16 CON).
void compute_coeff_kp(double con, double tol, int rk, double* coeff);
double zolo_fone(const double* coeff, int rk);
double zolo_next_con(double con, const double* coeff, int rk, double fone);
double hfunc(double x);
void qdwh_weights(double lowk, double* ak, double* bk, double* ck, double* lnext);

}  // namespace zolo
