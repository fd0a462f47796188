/* Oracle (test infrastructure): helpers shared by the C restatement's translation units. */
#ifndef CHQ_ORACLE_PORT_INTERNAL_H_
#define CHQ_ORACLE_PORT_INTERNAL_H_
double port_sign(double x);
double port_cfast(const double *s, double bn, double gamma);
double port_cflow(const double *s, double bn);
void port_pflux(const double *s, double bn, double gm1, double *e, double *pt, double f[7]);
#endif
