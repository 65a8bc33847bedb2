/* bam_nrharness.h -- oracle dump harness (test infrastructure) */
int nrharness_post_initialdata(tL *level);
int nrharness_post_evolve(tL *level);
