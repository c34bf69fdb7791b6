/* rdfSource/rdfRoutines/SRTMrdf.h -- TEST INFRASTRUCTURE ONLY: empty stand-in
 * (the RDF parser is not used by the reference's hot-path functions). */
