/* bam_nrgpu.h -- module header of the B200 evolution path for a BAM tree */
void bam_nrgpu(void);
