/* bam_nrgpu.h -- module header of the B200 evolution path for a BAM tree */
void bam_nrgpu(void);
/* the device multigrid for PickEllipticSolver (Punctures.c:283-311); the
 * argument list of multigrid() (multigrid.c:35) */
int nrgpu_multigrid(tL *level, tVarList *u, tVarList *f, tVarList *v, tVarList *c, int itmax, double tol,
                    double *normres, void (*lop)(tL *, tVarList *, tVarList *),
                    void (*lgs)(tL *, tVarList *, tVarList *));
